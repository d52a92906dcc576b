// Stand-in for the FemPIC app's field_solver.h (PETSc) when the app's generated main,
// apps_codegen/app_fempic_cg/fempic_opp.cpp, is built against this library: the oracle
// Makefile places it beside a build copy of that main as field_solver.h, so the main's
// #include "field_solver.h" finds the PETSc-free FESolver of the drop-in runtime.
#include "opp_fempic_solver.h"
