// Test infrastructure: linked into a generated main with -Wl,--wrap=_Z8opp_exitv (the mangled
// opp_exit()), so that the main's own opp_exit() first writes every dat, mesh and particle,
// with opp_print_dat_to_txtfile (prefix "final", suffix the dat's name) and then runs the
// library's opp_exit.  Compiled against whichever opp_lib.h the main is built with, so the same
// file serves the reference's seq backend and the drop-in runtime: a test compares the two
// runs' files.
#include "opp_lib.h"

extern "C" void __real__Z8opp_exitv();

extern "C" void __wrap__Z8opp_exitv() {
    for (opp_dat d : opp_dats)
        if (d && d->set) opp_print_dat_to_txtfile(d, "final", d->name);
    __real__Z8opp_exitv();
}
