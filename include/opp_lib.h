// opp_lib.h — the OP-PIC user API on the B200 backend (C++).
//
// Same names, argument meaning and error behaviour as the reference's
// opp_lib/include/opp_lib.h and opp_defs.h, so that a generated FemPIC main compiles and
// links against this library unchanged.  Storage: host copies AoS (as declared), device
// copies SoA [dim][capacity] as in the reference's CUDA backend.  All compute goes through
// the C ABI of oppb.h; errors abort through opp_abort as in the reference.
#pragma once

#include <cuda_runtime_api.h>

// The standard headers the reference's opp_lib.h brings in transitively (opp_defs.h,
// opp_util.h, opp_params.h, opp_profiler.h): app headers written against it, such as the
// FemPIC mesh loader, rely on them.
#include <algorithm>
#include <array>
#include <cfloat>
#include <chrono>
#include <cinttypes>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <random>
#include <sstream>
#include <stack>
#include <string>
#include <vector>

#include "oppb.h"

typedef int OPP_INT;
typedef double OPP_REAL;
typedef bool OPP_BOOL;
typedef std::string OPP_STRING;

#define MAX_CELL_INDEX INT_MAX
#define OPP_ROOT 0
#define OPP_DBG false

#define OPP_READ 0
#define OPP_WRITE 1
#define OPP_RW 2
#define OPP_INC 3
#define OPP_MIN 4
#define OPP_MAX 5

#define OPP_ARG_GBL 0
#define OPP_ARG_DAT 1
#define OPP_ARG_MAP 2

#define OPP_RUN_ON_ROOT(command) if (OPP_rank == OPP_ROOT command)
// Early returns of app functions on ranks outside the run (opp_defs.h:184-187).
#define OPP_RETURN_IF_INVALID_PROCESS if (OPP_rank < 0) return;
#define OPP_RETURN_ZERO_IF_INVALID_PROCESS if (OPP_rank < 0) return 0;
#define OPP_RETURN_EMPTY_IF_INVALID_PROCESS if (OPP_rank < 0) return "";

enum opp_iterate_type { OPP_ITERATE_ALL = 1, OPP_ITERATE_INJECTED };
enum opp_move_status { OPP_MOVE_DONE = 0, OPP_NEED_MOVE, OPP_NEED_REMOVE };
enum opp_data_type { DT_INT = 0, DT_REAL };
enum Dirty { NotDirty = 0, Device = 1, Host = 2 };
enum DeviceType { Device_CPU = 1, Device_GPU = 2 };
enum opp_reset { OPP_Reset_Core = 0, OPP_Reset_Set, OPP_Reset_ieh, OPP_Reset_inh, OPP_Reset_All };
enum opp_fill_type { OPP_HoleFill_All = 0, OPP_Sort_All, OPP_Shuffle_All, OPP_Sort_Periodic, OPP_Shuffle_Periodic };

struct opp_set_core;
typedef struct opp_set_core* opp_set;
struct opp_map_core;
typedef struct opp_map_core* opp_map;
struct opp_dat_core;
typedef struct opp_dat_core* opp_dat;

typedef int opp_access;
typedef int opp_arg_type;

struct opp_arg {
    int index;
    opp_dat dat;         // dataset
    opp_map map;         // indirect mapping
    opp_dat p2c_map;     // particle -> cell dat of a double-indirect access
    int dim;
    int idx;
    int size;
    char* data;          // host data
    char* data_d;        // device data
    int* map_data;       // host map
    int* map_data_d;     // device map (SoA)
    char const* type;
    opp_access acc;
    opp_arg_type argtype;
    int sent;
    int opt;
};

struct opp_set_core {
    int index;
    int size;                       // elements in the set
    char const* name;
    int core_size;
    int exec_size;
    int nonexec_size;
    bool is_particle;
    int set_capacity;               // allocated elements (particle sets)
    int diff;                       // particles added by the last increase
    int particle_size;              // bytes of one particle over all its dats
    opp_dat mesh_relation_dat = nullptr;
    std::vector<opp_dat>* particle_dats;
    int particle_remove_count;
    opp_set cells_set;
};

struct opp_map_core {
    int index;
    opp_set from;
    opp_set to;
    int dim;
    int* map;                       // host AoS [from.size][dim]
    int* map_d;                     // device SoA [dim][from.size]
    char const* name;
    int user_managed;
    opp_dat p2c_dat;                // particle maps: the mesh relation dat
};

struct opp_dat_core {
    int index;
    opp_set set;
    int dim;
    int size;                       // bytes of one element (dim * sizeof(type))
    char* data;                     // host AoS
    char* data_d;                   // device SoA [dim][stride]
    char* data_swap_d;              // device SoA, target of the cell sort
    char const* type;
    char const* name;
    int dirtybit;
    Dirty dirty_hd;                 // which copy is stale
    int user_managed;
    bool is_cell_index;
    opp_map p2c_map;
    uint64_t version;               // bumped whenever the device copy is written
};

struct opp_point {
    opp_point(double _x, double _y, double _z) : x(_x), y(_y), z(_z) {}
    opp_point() {}
    double x = 0.0, y = 0.0, z = 0.0;
};

constexpr double opp_zero_double16[16] = {0.0};
constexpr int opp_zero_int16[16] = {0};

namespace opp {

// `TYPE key = value` parameter file (the reference's opp::Params format): INT, REAL,
// BOOL, STRING; missing keys give INT_MAX / DBL_MAX / false / "NOT FOUND".
class Params {
   public:
    explicit Params(const std::string& file);
    Params() = default;
    template <typename T>
    T get(const std::string& key, bool error = true) const;
    template <typename T>
    void add(const std::string& key, T value);
    void write(std::FILE* out) const;

   private:
    std::map<std::string, std::string> ints_, reals_, bools_, strings_;
};

// Named wall-clock regions; device work is synchronised at region ends by the loops.
class Profiler {
   public:
    void reg(const std::string& name);
    void start(const std::string& name);
    void end(const std::string& name);
    double seconds(const std::string& name) const;
    long count(const std::string& name) const;
    void printProfile(bool all_ranks = false) const;

   private:
    struct Entry {
        double total = 0.0, started = 0.0;
        long count = 0;
    };
    std::map<std::string, Entry> entries_;
};

// Bounding box of the direct-hop grid (opp_lib/include/opp_direct_hop_core.h:41-177): the box of
// the node positions widened by `expansion`, computed by oppb_dh_bounding_box (3-D) or
// oppb_dh_bounding_box_2d (2-D: z stays 0) exactly as the reference does.  One unpartitioned
// mesh: the global box is the local one.
class BoundingBox {
   public:
    BoundingBox(const opp_dat node_pos_dat, int dim, const opp_point expansion);
    BoundingBox(int dim, opp_point min_coordinate, opp_point max_coordinate);
    const opp_point& getLocalMin() const { return box_[0]; }
    const opp_point& getLocalMax() const { return box_[1]; }
    const opp_point& getGlobalMin() const { return box_[0]; }
    const opp_point& getGlobalMax() const { return box_[1]; }
    int getDim() const { return dim_; }
    // The node positions the box was made from (nullptr for a box given by its corners); the
    // grid build bins the cells with them.
    opp_dat nodePositions() const { return node_pos_; }
    opp_point domain_expansion;

   private:
    int dim_ = 0;
    opp_point box_[2];
    opp_dat node_pos_ = nullptr;
};

}  // namespace opp

extern std::unique_ptr<opp::Params> opp_params;
extern std::unique_ptr<opp::Profiler> opp_profiler;

extern int OPP_rank;
extern int OPP_comm_size;
extern int OPP_main_loop_iter;
extern int OPP_comm_iteration;
extern int OPP_fill_period;
extern opp_fill_type OPP_fill_type;
extern double OPP_part_alloc_mult;
extern int OPP_iter_start;
extern int OPP_iter_end;
extern int OPP_move_max_hops;       // the parameter file's opp_move_max_hops, else -1 (unbounded there)
// Communication and hop statistics the apps' logs print (opp_defs.h:428-439); one GPU has no
// communication rounds, so they stay 0.
extern int OPP_max_comm_iteration;
extern int OPP_part_comm_count_per_iter;
extern int OPP_move_moreX_hops;
// The rest of opp_defs.h:417-450 with the reference's defaults (opp_lib_core.cpp:45-69).
// OPP_maps_base_index = 1 makes opp_decl_map take 1-based maps (each entry less 1 on
// declaration); OPP_gpu_threads_per_block holds the parameter file's opp_threads_per_block and
// OPP_gpu_direct its opp_gpu_direct (informational: the kernels' launch shapes come from
// oppb_tuning); OPP_mpi_part_alloc_mult and OPP_dh_data_dump are set from the command line
// (OPP_MPI_ALLOC_MULT=, OPP_DH_DATA_DUMP=) as there; the others stay at their one-rank values.
extern double OPP_hybrid_balance;
extern int OPP_maps_base_index;
extern int OPP_auto_soa;
extern int OPP_gpu_direct;
extern int OPP_mpi_part_alloc_mult;
extern int* OPP_mesh_relation_data;
extern int* OPP_mesh_relation_data_d;
extern int OPP_gpu_threads_per_block;
extern size_t OPP_gpu_shared_mem_per_block;
extern int OPP_part_cells_set_size;
extern bool OPP_dh_data_dump;
extern bool useGlobalMove;  // set by opp_init_direct_hop_cg when opp_global_move is on
extern size_t opp_maxSavedDHGrid[3];
extern size_t opp_minSavedDHGrid[3];
extern std::vector<opp_set> opp_sets;
extern std::vector<opp_map> opp_maps;
extern std::vector<opp_dat> opp_dats;

// ------------------------------------------------------------------ lifetime
void opp_init(int argc, char** argv);
void opp_exit();
void opp_abort(std::string s = "");
void opp_printf(const char* function, const char* format, ...);

// -------------------------------------------------------------- declarations
opp_set opp_decl_set(int size, char const* name);
opp_set opp_decl_particle_set(int size, char const* name, opp_set cells_set);
opp_set opp_decl_particle_set(char const* name, opp_set cells_set);
opp_map opp_decl_map(opp_set from, opp_set to, int dim, int* imap, char const* name);
opp_dat opp_decl_dat(opp_set set, int dim, opp_data_type dtype, void* data, char const* name);
// From a text file: a "size dim" header, then `size` rows of `dim` values (at least the set's
// size rows; dim 1-4 for int, 1-4 or 16 for double), as opp_load_from_file_core reads it
// (opp_lib/src/core/opp_lib_file_core.cpp:180-281; opp_lib/src/cuda/opp_cuda.cu:361-385).
// A missing or malformed file ends the program with status -1, as there.
opp_map opp_decl_map_txt(opp_set from, opp_set to, int dim, const char* file_name, char const* name);
opp_dat opp_decl_dat_txt(opp_set set, int dim, opp_data_type dtype, const char* file_name, char const* name);

void opp_decl_const_impl(int dim, int size, char* data, const char* name);
template <typename T>
void opp_decl_const(int dim, T* data, const char* name) {
    opp_decl_const_impl(dim, sizeof(T), (char*)data, name);
}
// Value of a constant registered with opp_decl_const (abort if unknown).
// Element `index` of a constant declared by opp_decl_const (B200 extension: the generated loops
// of this library read their constants here).
double opp_get_const(const char* name, int index = 0);

// ------------------------------------------------------------------- args
opp_arg opp_arg_gbl(double* data, int dim, char const* typ, opp_access acc);
opp_arg opp_arg_gbl(int* data, int dim, char const* typ, opp_access acc);
opp_arg opp_arg_gbl(const bool* data, int dim, char const* typ, opp_access acc);

opp_arg opp_arg_dat(opp_dat dat, int idx, opp_map map, int dim, const char* typ, opp_map p2c_map, opp_access acc,
                    bool offset = true);
opp_arg opp_arg_dat(opp_dat dat, int idx, opp_map map, opp_map p2c_map, opp_access acc, bool offset = true);
opp_arg opp_arg_dat(opp_dat dat, int idx, opp_map map, opp_access acc, bool offset = true);
opp_arg opp_arg_dat(opp_dat dat, opp_map p2c_map, opp_access acc, bool offset = true);
opp_arg opp_arg_dat(opp_dat dat, opp_access acc, bool offset = true);
opp_arg opp_arg_dat(opp_map data_map, opp_access acc, bool offset = true);
opp_arg opp_arg_dat(opp_map data_map, opp_map p2c_map, opp_access acc, bool offset = true);
opp_arg opp_arg_dat(opp_map data_map, int idx, opp_map map, opp_access acc, bool offset = true);
opp_arg opp_arg_dat(opp_map data_map, int idx, opp_map map, opp_map p2c_map, opp_access acc, bool offset = true);

// -------------------------------------------------------------- particles
void opp_increase_particle_count(opp_set part_set, int insert_count);
void opp_inc_part_count_with_distribution(opp_set part_set, int insert_count, opp_dat part_dist,
                                          bool calc_new = true);
void opp_reset_num_particles_to_insert(opp_set set);
void opp_init_particle_move(opp_set set, int nargs, opp_arg* args);
bool opp_finalize_particle_move(opp_set set);
void opp_particle_sort(opp_set set);

void opp_reset_dat_impl(opp_dat dat, char* val, opp_reset reset = OPP_Reset_All);
template <typename T>
void opp_reset_dat(opp_dat dat, T* val, opp_reset reset = OPP_Reset_All) {
    opp_reset_dat_impl(dat, (char*)val, reset);
}

// --------------------------------------------------------------- transfers
void opp_upload_dat(opp_dat dat);
void opp_download_dat(opp_dat dat);
void opp_download_particle_set(opp_set set, bool force_download = false);
void opp_upload_particle_set(opp_set set, bool realloc = false);
template <typename T>
T* opp_get_data(opp_dat dat) {
    opp_download_dat(dat);
    return (T*)dat->data;
}
OPP_INT* opp_get_data(opp_map map);
// Text dumps in the reference CUDA backend's format and place (opp_lib/src/cuda/opp_cuda.cu:458-481,
// opp_lib/src/core/opp_lib_file_core.cpp:35-178): files/<prefix>_cuda_<suffix> for a dat and
// files/<prefix>_cuda0__<suffix> for a map, a "size dim -- exec nonexec" header, one row per
// element (" %2.25lE" per double, -0 written, and left in the host copy, as +0; " %d" per
// int), then the two import_exec_below / import_non_exec_below marker lines.  A file that
// cannot be opened ends the program with status 2, as there.
void opp_print_dat_to_txtfile(opp_dat dat, const char* file_prefix, const char* file_suffix);
void opp_print_map_to_txtfile(opp_map map, const char* file_prefix, const char* file_suffix);
// The dat's values on stdout (opp_dump_dat_core, opp_lib_file_core.cpp:103-131): "\t %+2.25lE"
// per double and a "\t\n" per row.  The reference names its other dump types "real" and
// "integer", so an int dat ends the program there (message, status 0); it does here too.
void opp_dump_dat(opp_dat data);
// The dat with its host copy current (opp_cuda.cu:484-499); particle dats are refused.
opp_dat opp_fetch_data(opp_dat dat);

// One-GPU build: halo exchanges, double-indirect reductions and mesh colouring are identities
// (the reference defines them only for MPI builds, opp_lib/src/mpi/).
int opp_mpi_halo_exchanges_grouped(opp_set set, int nargs, opp_arg* args, DeviceType device);
int opp_mpi_halo_exchanges(opp_set set, int nargs, opp_arg* args);
void opp_mpi_halo_exchange(opp_arg* arg, int exec_flag);
void opp_mpi_halo_wait_all(int nargs, opp_arg* args);
void opp_mpi_force_halo_update_if_dirty(opp_set set, std::vector<opp_dat> dats, DeviceType device);
void opp_set_dirtybit_grouped(int nargs, opp_arg* args, DeviceType device);
// An OPP_INC through a particle's cell map (opp_lib/src/mpi/opp_mpi_utils.cpp:537-544).
bool is_double_indirect_reduction(opp_arg& arg);
void opp_init_double_indirect_reductions(int nargs, opp_arg* args);
void opp_exchange_double_indirect_reductions(int nargs, opp_arg* args);
void opp_complete_double_indirect_reductions(int nargs, opp_arg* args);
void opp_colour_cartesian_mesh(const int ndim, std::vector<int> cell_counts, opp_dat cell_index,
                               const opp_dat cell_colors, const int cell_ghosts = 0);
inline int64_t opp_get_global_value(int64_t value) { return value; }
// Sum, maximum and minimum over ranks (opp_util.h:274): on one GPU, the value three times.
inline void opp_get_global_values(const int64_t value, int64_t& gbl_value, int64_t& gbl_max, int64_t& gbl_min) {
    gbl_value = gbl_max = gbl_min = value;
}

// Particle initialisation helpers of opp_util.h:108-175, used by the apps' host set-up: the
// same draws in the same order from the caller's engine, so a seeded set-up gives the
// reference's particles.  Per dimension, N draws of N(mu, sigma).
template <typename RNG>
inline std::vector<std::vector<double>> get_normal_distribution(const int N, const int ndim, const double mu,
                                                                const double sigma, RNG& rng) {
    std::normal_distribution<> normal{mu, sigma};
    std::vector<std::vector<double>> out(ndim, std::vector<double>(N));
    for (int d = 0; d < ndim; d++)
        for (int p = 0; p < N; p++) out[d][p] = normal(rng);
    return out;
}

// Per dimension d, N draws of extents[d] * U[0, 1).
template <typename RNG>
inline std::vector<std::vector<double>> get_uniform_within_extents(const int N, const int ndim, const double* extents,
                                                                   RNG& rng) {
    std::uniform_real_distribution<double> unit(0.0, 1.0);
    std::vector<std::vector<double>> out(ndim, std::vector<double>(N));
    for (int d = 0; d < ndim; d++)
        for (int p = 0; p < N; p++) out[d][p] = extents[d] * unit(rng);
    return out;
}

// npart_per_cell particles in each cell c: cell c, position cell_pos_ll[c] plus a draw of
// get_uniform_within_extents (cells in order).  The engine is taken by value, as there.
template <typename T>
inline void uniform_within_cartesian_cells(int ndim, const double* extents, const T* cell_pos_ll,
                                           const int64_t cells_set_size, const int64_t npart_per_cell,
                                           std::vector<std::vector<double>>& positions, std::vector<int>& cells,
                                           std::mt19937 rng) {
    const int64_t total = npart_per_cell * cells_set_size;
    cells.resize(total);
    positions.resize(ndim);
    for (int d = 0; d < ndim; d++) positions[d] = std::vector<double>(total);
    for (int64_t c = 0; c < cells_set_size; c++) {
        const auto local = get_uniform_within_extents((int)npart_per_cell, ndim, extents, rng);
        for (int64_t k = 0; k < npart_per_cell; k++) {
            const int64_t p = c * npart_per_cell + k;
            cells.at(p) = (int)c;
            for (int d = 0; d < ndim; d++) positions.at(d).at(p) = cell_pos_ll[c * ndim + d] + local.at(d).at(k);
        }
    }
}

// printf-formatted value (opp_util.h:85).
template <typename T>
std::string str(T value, std::string format) {
    char buf[64];
    std::snprintf(buf, sizeof buf, format.c_str(), value);
    return std::string(buf);
}

// --------------------------------------------------------- B200 extensions
// Device-resident packed mesh and scratch shared by the generated-loop entry points.
namespace oppb_rt {
cudaStream_t stream();
// Bound on the cell visits of one particle's walk: OPP_move_max_hops when positive, else 4096.
int max_hops();
// The number of opp_init calls so far: a cache keyed on a set, dat or map pointer also keeps the
// generation it was made in, since after opp_exit and a new opp_init a new object may reuse an
// old one's address.
int generation();
const oppb_tet_mesh& tet_mesh(opp_dat c_det, opp_dat c_volume, opp_map c2c, opp_map c2n, opp_dat c_ef);
void* workspace(size_t bytes);
oppb_move_status* move_status();
uint32_t* remove_bits(opp_set set);
void mark_device_written(opp_dat dat);
void sync_host_to_device(opp_dat dat);
}  // namespace oppb_rt
