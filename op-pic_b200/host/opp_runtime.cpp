// The opp_* runtime on one B200: registry of sets, maps and dats, device storage in the
// reference CUDA backend's layout (SoA [dim][capacity]), particle set growth on the device,
// the move finalize (hole fill or cell sort), transfers, parameters and the profiler.
// Every kernel launch goes through the C ABI of oppb.h; this file only allocates and
// sequences.  Errors abort through opp_abort, as the reference does.

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cstring>
#include <fstream>
#include <sstream>

#include "opp_lib.h"
#include "oppb_dh.h"

std::unique_ptr<opp::Params> opp_params;
std::unique_ptr<opp::Profiler> opp_profiler;
int OPP_rank = 0;
int OPP_comm_size = 1;
int OPP_main_loop_iter = 0;
int OPP_comm_iteration = 0;
int OPP_max_comm_iteration = 0;
int OPP_part_comm_count_per_iter = 0;
int OPP_move_moreX_hops = -1;
int OPP_fill_period = 2;
opp_fill_type OPP_fill_type = OPP_HoleFill_All;
double OPP_part_alloc_mult = 1.0;
int OPP_iter_start = 0;
int OPP_iter_end = 0;
// The reference's -1 leaves its walks unbounded; the kernels here stop a walk after
// oppb_rt::max_hops() cell visits (this value when positive, set by opp_move_max_hops in the
// parameter file, else 4096) and report OPPB_ERR_HOP_LIMIT.
int OPP_move_max_hops = -1;
double OPP_hybrid_balance = 1.0;
int OPP_maps_base_index = 0;
int OPP_auto_soa = 1;  // device dats are SoA, as the CUDA backend sets it in opp_init
int OPP_gpu_direct = 0;
int OPP_mpi_part_alloc_mult = 1;
int* OPP_mesh_relation_data = nullptr;
int* OPP_mesh_relation_data_d = nullptr;
int OPP_gpu_threads_per_block = 32;  // OPP_DEFAULT_GPU_THREADS_PER_BLOCK
size_t OPP_gpu_shared_mem_per_block = 0;
int OPP_part_cells_set_size = 0;
bool OPP_dh_data_dump = false;
bool useGlobalMove = false;
size_t opp_maxSavedDHGrid[3];
size_t opp_minSavedDHGrid[3];
std::vector<opp_set> opp_sets;
std::vector<opp_map> opp_maps;
std::vector<opp_dat> opp_dats;

namespace {

int g_generation = 0;  // opp_init calls so far: caches keyed on sets, dats or maps check it

struct Runtime {
    cudaStream_t stream = nullptr;
    std::map<std::string, std::vector<double>> consts;
    void* ws = nullptr;
    size_t ws_bytes = 0;
    oppb_move_status* status = nullptr;
    std::map<opp_set, std::pair<uint32_t*, size_t>> bits;
    // Packed mesh and the inputs it was packed from (dat versions).
    struct {
        opp_dat det = nullptr, vol = nullptr, ef = nullptr;
        opp_map c2c = nullptr, c2n = nullptr;
        uint64_t det_v = 0, vol_v = 0, ef_v = 0;
        oppb_tet_mesh m{};
    } mesh;
    int32_t* invalid = nullptr;
};

Runtime& rt() {
    static Runtime r;
    return r;
}

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) opp_abort(std::string(what) + ": " + cudaGetErrorString(e));
}

void check_oppb(int rc, const char* what) {
    if (rc != OPPB_OK) opp_abort(std::string(what) + ": " + oppb_status_string(rc));
}

char* dev_alloc(size_t bytes) {
    void* p = nullptr;
    check_cuda(cudaMalloc(&p, bytes ? bytes : 16), "cudaMalloc");
    return static_cast<char*>(p);
}

void dev_free(void* p) {
    if (p) cudaFree(p);
}

char* copy_name(const char* s) {
    const size_t n = std::strlen(s);
    char* c = static_cast<char*>(std::malloc(n + 1));
    std::memcpy(c, s, n + 1);
    return c;
}

int stride_of(opp_set set) { return set->is_particle ? std::max(set->set_capacity, 1) : std::max(set->size, 1); }

int elem_bytes(opp_dat dat) { return dat->size / dat->dim; }

// Host AoS [n][dim] <-> device SoA [dim][stride], first n elements.
void upload(opp_dat dat, int n) {
    if (!dat->data || n <= 0) return;
    const int eb = elem_bytes(dat), dim = dat->dim, stride = stride_of(dat->set);
    std::vector<char> soa((size_t)dim * n * eb);
    for (int i = 0; i < n; i++)
        for (int d = 0; d < dim; d++)
            std::memcpy(&soa[((size_t)d * n + i) * eb], dat->data + ((size_t)i * dim + d) * eb, eb);
    check_cuda(cudaMemcpy2DAsync(dat->data_d, (size_t)stride * eb, soa.data(), (size_t)n * eb, (size_t)n * eb, dim,
                                 cudaMemcpyHostToDevice, rt().stream),
               "upload");
    check_cuda(cudaStreamSynchronize(rt().stream), "upload sync");
}

void download(opp_dat dat, int n) {
    if (n <= 0) return;
    const int eb = elem_bytes(dat), dim = dat->dim, stride = stride_of(dat->set);
    std::vector<char> soa((size_t)dim * n * eb);
    check_cuda(cudaMemcpy2DAsync(soa.data(), (size_t)n * eb, dat->data_d, (size_t)stride * eb, (size_t)n * eb, dim,
                                 cudaMemcpyDeviceToHost, rt().stream),
               "download");
    check_cuda(cudaStreamSynchronize(rt().stream), "download sync");
    for (int i = 0; i < n; i++)
        for (int d = 0; d < dim; d++)
            std::memcpy(dat->data + ((size_t)i * dim + d) * eb, &soa[((size_t)d * n + i) * eb], eb);
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

// ------------------------------------------------------------------ params

namespace opp {

Params::Params(const std::string& file) {
    std::ifstream in(file);
    if (!in) opp_abort("cannot open parameter file " + file);
    std::string line;
    while (std::getline(in, line)) {
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        std::istringstream ls(line);
        std::string type, key, eq, value;
        if (!(ls >> type >> key >> eq) || eq != "=") continue;
        std::getline(ls, value);
        const size_t a = value.find_first_not_of(" \t"), b = value.find_last_not_of(" \t\r");
        value = (a == std::string::npos) ? "" : value.substr(a, b - a + 1);
        if (type == "INT") ints_[key] = value;
        else if (type == "REAL") reals_[key] = value;
        else if (type == "BOOL") bools_[key] = value;
        else if (type == "STRING") strings_[key] = value;
    }
}

template <>
OPP_INT Params::get<OPP_INT>(const std::string& key, bool) const {
    auto it = ints_.find(key);
    return it == ints_.end() ? INT_MAX : std::stoi(it->second);
}
template <>
OPP_REAL Params::get<OPP_REAL>(const std::string& key, bool) const {
    auto it = reals_.find(key);
    return it == reals_.end() ? DBL_MAX : std::stod(it->second);
}
template <>
OPP_BOOL Params::get<OPP_BOOL>(const std::string& key, bool) const {
    auto it = bools_.find(key);
    return it != bools_.end() && (it->second == "true" || it->second == "1");
}
template <>
OPP_STRING Params::get<OPP_STRING>(const std::string& key, bool) const {
    auto it = strings_.find(key);
    return it == strings_.end() ? std::string("NOT FOUND") : it->second;
}
template <>
void Params::add<OPP_INT>(const std::string& key, OPP_INT v) { ints_[key] = std::to_string(v); }
template <>
void Params::add<OPP_REAL>(const std::string& key, OPP_REAL v) {
    std::ostringstream s;
    s.precision(17);
    s << v;
    reals_[key] = s.str();
}
template <>
void Params::add<OPP_BOOL>(const std::string& key, OPP_BOOL v) { bools_[key] = v ? "true" : "false"; }
template <>
void Params::add<OPP_STRING>(const std::string& key, OPP_STRING v) { strings_[key] = v; }

void Params::write(std::FILE* out) const {
    for (auto& kv : ints_) std::fprintf(out, "INT %s = %s\n", kv.first.c_str(), kv.second.c_str());
    for (auto& kv : reals_) std::fprintf(out, "REAL %s = %s\n", kv.first.c_str(), kv.second.c_str());
    for (auto& kv : bools_) std::fprintf(out, "BOOL %s = %s\n", kv.first.c_str(), kv.second.c_str());
    for (auto& kv : strings_) std::fprintf(out, "STRING %s = %s\n", kv.first.c_str(), kv.second.c_str());
}

void Profiler::reg(const std::string& name) { entries_[name]; }
void Profiler::start(const std::string& name) { entries_[name].started = now_s(); }
void Profiler::end(const std::string& name) {
    auto& e = entries_[name];
    e.total += now_s() - e.started;
    e.count++;
}
double Profiler::seconds(const std::string& name) const {
    auto it = entries_.find(name);
    return it == entries_.end() ? 0.0 : it->second.total;
}
long Profiler::count(const std::string& name) const {
    auto it = entries_.find(name);
    return it == entries_.end() ? 0 : it->second.count;
}
void Profiler::printProfile(bool) const {
    std::printf("%-40s %10s %14s\n", "profile", "count", "seconds");
    for (auto& kv : entries_) std::printf("%-40s %10ld %14.6f\n", kv.first.c_str(), kv.second.count, kv.second.total);
}

}  // namespace opp

// ---------------------------------------------------------------- lifetime

void opp_printf(const char* function, const char* format, ...) {
    char buf[4096];
    va_list args;
    va_start(args, format);
    std::vsnprintf(buf, sizeof buf, format, args);
    va_end(args);
    std::printf("%s[%d][%d] - %s\n", function, OPP_rank, OPP_main_loop_iter, buf);
}

void opp_abort(std::string s) {
    std::fprintf(stderr, "opp_abort: %s\n", s.c_str());
    std::exit(-1);
}

void opp_init(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "Usage: %s <config_file> ...\n", argc > 0 ? argv[0] : "app");
        std::exit(-1);
    }
    opp_sets.clear();
    opp_maps.clear();
    opp_dats.clear();
    opp_params = std::make_unique<opp::Params>(argv[1]);
    opp_profiler = std::make_unique<opp::Profiler>();
    const double mult = opp_params->get<OPP_REAL>("opp_allocation_multiple");
    OPP_part_alloc_mult = (mult == DBL_MAX) ? 1.0 : mult;
    const std::string fill = opp_params->get<OPP_STRING>("opp_fill");
    const int period = opp_params->get<OPP_INT>("opp_fill_period");
    // opp_init's parse (opp_lib/src/core/opp_lib_core.cpp:86-101); a value it does not know is
    // refused here, where the reference would keep its default silently.
    if (fill == "HoleFill_All" || fill == "NOT FOUND") OPP_fill_type = OPP_HoleFill_All;
    else if (fill == "Sort_All") OPP_fill_type = OPP_Sort_All;
    else if (fill == "Shuffle_All") OPP_fill_type = OPP_Shuffle_All;
    else if (fill == "Sort_Periodic") OPP_fill_type = OPP_Sort_Periodic;
    else if (fill == "Shuffle_Periodic") OPP_fill_type = OPP_Shuffle_Periodic;
    else opp_abort("opp_fill " + fill + " is not a fill type");
    // A missing opp_fill_period reads as INT_MAX, which the reference takes as the period too.
    if ((OPP_fill_type == OPP_Sort_Periodic || OPP_fill_type == OPP_Shuffle_Periodic) && period >= 0)
        OPP_fill_period = period;
    const int hops = opp_params->get<OPP_INT>("opp_move_max_hops");
    if (hops != INT_MAX && hops > 0) OPP_move_max_hops = hops;
    // B200 extension (absent from the reference's parameter files, default false): node-charge
    // deposits with order-independent integer sums, bit-identical from run to run.
    if (opp_params->get<OPP_BOOL>("oppb_deterministic_deposit")) {
        oppb_tuning t{};
        oppb_get_tuning(&t);
        t.deposit = OPPB_DEPOSIT_EXACT;
        if (oppb_set_tuning(&t) != OPPB_OK) opp_abort("oppb_set_tuning");
    }
    const int tpb = opp_params->get<OPP_INT>("opp_threads_per_block");
    if (tpb > 0 && tpb < INT_MAX) OPP_gpu_threads_per_block = tpb;
    const int gpu_direct = opp_params->get<OPP_INT>("opp_gpu_direct");
    if (gpu_direct > 0 && gpu_direct < INT_MAX) OPP_gpu_direct = gpu_direct;
    // opp_set_args_core (opp_lib_core.cpp:149-184): the first of its keys an argument holds.
    for (int n = 1; n < argc; n++) {
        char tmp[64] = {0};
        if (const char* p = std::strstr(argv[n], "OPP_ALLOC_MULT=")) {
            std::strncpy(tmp, p, 17);
            OPP_part_alloc_mult = std::atof(tmp + 15);
        } else if (const char* q = std::strstr(argv[n], "OPP_MPI_ALLOC_MULT=")) {
            std::strncpy(tmp, q, 21);
            OPP_mpi_part_alloc_mult = std::atoi(tmp + 19);
        } else if (const char* r = std::strstr(argv[n], "OPP_DH_DATA_DUMP=")) {
            std::strncpy(tmp, r, 18);
            OPP_dh_data_dump = std::atoi(tmp + 17) != 0;
        }
    }
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) opp_abort("no CUDA device");
    check_cuda(cudaSetDevice(0), "cudaSetDevice");
    cudaDeviceProp prop{};
    check_cuda(cudaGetDeviceProperties(&prop, 0), "cudaGetDeviceProperties");
    OPP_gpu_shared_mem_per_block = prop.sharedMemPerBlock;
    check_cuda(cudaStreamCreateWithFlags(&rt().stream, cudaStreamNonBlocking), "stream");
    rt().status = reinterpret_cast<oppb_move_status*>(dev_alloc(sizeof(oppb_move_status)));
    ++g_generation;
    rt().invalid = reinterpret_cast<int32_t*>(dev_alloc(sizeof(int32_t)));
}

void opp_exit() {
    if (opp_profiler && opp_params && opp_params->get<OPP_BOOL>("opp_profile_all")) opp_profiler->printProfile();
    cudaStreamSynchronize(rt().stream);
    for (opp_dat d : opp_dats) {
        dev_free(d->data_d);
        dev_free(d->data_swap_d);
        std::free(d->data);
        std::free((char*)d->name);
        delete d;
    }
    for (opp_map m : opp_maps) {
        dev_free(m->map_d);
        std::free(m->map);
        std::free((char*)m->name);
        delete m;
    }
    for (opp_set s : opp_sets) {
        delete s->particle_dats;
        std::free((char*)s->name);
        delete s;
    }
    opp_sets.clear();
    opp_maps.clear();
    opp_dats.clear();
    auto& r = rt();
    for (auto& kv : r.bits) dev_free(kv.second.first);
    r.bits.clear();
    dev_free(r.ws);
    dev_free(r.status);
    dev_free(r.invalid);
    dev_free(r.mesh.m.det);
    dev_free(r.mesh.m.nav);
    dev_free(r.mesh.m.c2n);
    dev_free(r.mesh.m.ef);
    r.ws = nullptr;
    r.ws_bytes = 0;
    r.status = nullptr;
    r.mesh = {};
    if (r.stream) cudaStreamDestroy(r.stream);
    r.stream = nullptr;
}

// ------------------------------------------------------------ declarations

opp_set opp_decl_set(int size, char const* name) {
    opp_set s = new opp_set_core{};
    s->index = (int)opp_sets.size();
    s->size = size;
    s->core_size = size;
    s->name = copy_name(name);
    s->is_particle = false;
    s->set_capacity = size;
    s->particle_dats = new std::vector<opp_dat>();
    s->cells_set = nullptr;
    opp_sets.push_back(s);
    return s;
}

opp_set opp_decl_particle_set(int size, char const* name, opp_set cells_set) {
    opp_set s = opp_decl_set(0, name);
    s->is_particle = true;
    s->cells_set = cells_set;
    s->set_capacity = 0;
    if (size > 0) {
        s->size = 0;
        opp_increase_particle_count(s, size);
        s->diff = 0;
    }
    return s;
}

opp_set opp_decl_particle_set(char const* name, opp_set cells_set) { return opp_decl_particle_set(0, name, cells_set); }

namespace {
opp_dat new_dat(opp_set set, int dim, const char* type, int elem, const char* name) {
    opp_dat d = new opp_dat_core{};
    d->index = (int)opp_dats.size();
    d->set = set;
    d->dim = dim;
    d->size = dim * elem;
    d->type = type;
    d->name = copy_name(name);
    d->dirty_hd = NotDirty;
    d->version = 1;
    const size_t cap = (size_t)stride_of(set);
    d->data = static_cast<char*>(std::calloc(cap, (size_t)d->size));
    d->data_d = dev_alloc(cap * d->size);
    check_cuda(cudaMemsetAsync(d->data_d, 0, cap * d->size, rt().stream), "memset");
    if (set->is_particle) {
        d->data_swap_d = dev_alloc(cap * d->size);
        set->particle_dats->push_back(d);
    }
    opp_dats.push_back(d);
    return d;
}
}  // namespace

opp_dat opp_decl_dat(opp_set set, int dim, opp_data_type dtype, void* data, char const* name) {
    const bool is_int = (dtype == DT_INT);
    opp_dat d = new_dat(set, dim, is_int ? "int" : "double", is_int ? 4 : 8, name);
    if (data) {
        std::memcpy(d->data, data, (size_t)set->size * d->size);
        upload(d, set->size);
    }
    return d;
}

namespace {
// `rows` rows of `dim` values from a text file with a "size dim" header (size >= rows), as
// opp_load_from_file_core reads it: the dims it has formats for (int 1-4, double 1-4 and 16);
// a missing file, a header that does not fit or a value that does not parse ends the program
// with status -1 after the reference's message.
std::vector<char> load_txt(const char* file_name, int rows, int dim, bool is_double) {
    std::FILE* fp = std::fopen(file_name, "r");
    if (!fp) {
        std::printf("\topp_load_from_file - Unable to open file %s\n", file_name);
        std::exit(-1);
    }
    int fsize = -1, fdim = -1;
    if (std::fscanf(fp, "%d %d\n", &fsize, &fdim) != 2) {
        std::printf("\topp_load_from_file - error reading file data from %s\n", file_name);
        std::exit(-1);
    }
    if (fsize < rows || fdim != dim) {
        std::printf("\topp_load_from_file - dim and/or set_size issue in file %s\n", file_name);
        std::exit(-1);
    }
    const bool dim_ok = (dim >= 1 && dim <= 4) || (is_double && dim == 16);
    std::vector<char> out((size_t)std::max(rows, 1) * std::max(dim, 1) * (is_double ? 8 : 4));
    for (int n = 0; n < rows; n++) {
        bool ok = dim_ok;
        for (int j = 0; ok && j < dim; j++) {
            const size_t k = (size_t)n * dim + j;
            ok = is_double ? std::fscanf(fp, " %lf", reinterpret_cast<double*>(out.data()) + k) == 1
                           : std::fscanf(fp, " %d", reinterpret_cast<int*>(out.data()) + k) == 1;
        }
        if (!ok) {
            opp_printf("opp_load_from_file", "Error reading %s from %s at index %d", is_double ? "Double" : "Int",
                       file_name, n);
            std::exit(-1);
        }
    }
    std::fclose(fp);
    return out;
}
}  // namespace

opp_dat opp_decl_dat_txt(opp_set set, int dim, opp_data_type dtype, const char* file_name, char const* name) {
    std::vector<char> v = load_txt(file_name, set->size, dim, dtype != DT_INT);
    return opp_decl_dat(set, dim, dtype, v.data(), name);
}

opp_map opp_decl_map_txt(opp_set from, opp_set to, int dim, const char* file_name, char const* name) {
    std::vector<char> v = load_txt(file_name, from->size, dim, false);
    return opp_decl_map(from, to, dim, reinterpret_cast<int*>(v.data()), name);
}

opp_map opp_decl_map(opp_set from, opp_set to, int dim, int* imap, char const* name) {
    // A 1-based map (OPP_maps_base_index = 1) is taken 0-based, as opp_decl_map_core does
    // (opp_lib/src/core/opp_lib_core.cpp:261-264); the caller's array is not changed.
    std::vector<int> rebased;
    if (imap && OPP_maps_base_index == 1) {
        rebased.assign(imap, imap + (size_t)from->size * dim);
        for (int& v : rebased) v--;
        imap = rebased.data();
    }
    opp_map m = new opp_map_core{};
    m->index = (int)opp_maps.size();
    m->from = from;
    m->to = to;
    m->dim = dim;
    m->name = copy_name(name);
    if (from->is_particle) {
        // A particle map is the particle set's mesh relation dat (opp_lib_core.cpp:272-286).
        opp_dat d = new_dat(from, dim, "int", 4, name);
        d->is_cell_index = true;
        d->p2c_map = m;
        from->mesh_relation_dat = d;
        m->p2c_dat = d;
        const size_t cap = (size_t)stride_of(from) * dim;
        check_oppb(oppb_fill(d->data_d, (int64_t)cap, 4, (uint32_t)MAX_CELL_INDEX, rt().stream), "fill");
        for (size_t i = 0; i < cap; i++) reinterpret_cast<int*>(d->data)[i] = MAX_CELL_INDEX;
        if (imap && from->size > 0) {
            std::memcpy(d->data, imap, (size_t)from->size * dim * sizeof(int));
            upload(d, from->size);
        }
    } else {
        const size_t n = (size_t)from->size * dim;
        m->map = static_cast<int*>(std::malloc(std::max<size_t>(n, 1) * sizeof(int)));
        if (imap) std::memcpy(m->map, imap, n * sizeof(int));
        std::vector<int> soa(std::max<size_t>(n, 1));
        for (int i = 0; i < from->size; i++)
            for (int k = 0; k < dim; k++) soa[(size_t)k * from->size + i] = m->map[(size_t)i * dim + k];
        m->map_d = reinterpret_cast<int*>(dev_alloc(std::max<size_t>(n, 1) * sizeof(int)));
        check_cuda(cudaMemcpy(m->map_d, soa.data(), n * sizeof(int), cudaMemcpyHostToDevice), "map upload");
    }
    opp_maps.push_back(m);
    return m;
}

void opp_decl_const_impl(int dim, int size, char* data, const char* name) {
    std::vector<double> v((size_t)dim);
    for (int i = 0; i < dim; i++) {
        if (size == sizeof(double)) v[i] = reinterpret_cast<double*>(data)[i];
        else if (size == sizeof(int)) v[i] = reinterpret_cast<int*>(data)[i];
        else opp_abort(std::string("opp_decl_const: unsupported element size for ") + name);
    }
    rt().consts[name] = v;
}

double opp_get_const(const char* name, int index) {
    auto it = rt().consts.find(name);
    if (it == rt().consts.end() || index < 0 || (size_t)index >= it->second.size())
        opp_abort(std::string("unknown const ") + name);
    return it->second[(size_t)index];
}

// -------------------------------------------------------------------- args

opp_arg opp_arg_gbl(double* data, int dim, char const* typ, opp_access acc) {
    opp_arg a{};
    a.argtype = OPP_ARG_GBL;
    a.dim = dim;
    a.idx = -1;
    a.size = dim * (int)sizeof(double);
    a.data = (char*)data;
    a.type = typ;
    a.acc = acc;
    a.opt = 1;
    return a;
}
opp_arg opp_arg_gbl(int* data, int dim, char const* typ, opp_access acc) {
    opp_arg a = opp_arg_gbl((double*)nullptr, dim, typ, acc);
    a.size = dim * (int)sizeof(int);
    a.data = (char*)data;
    return a;
}
opp_arg opp_arg_gbl(const bool* data, int dim, char const* typ, opp_access acc) {
    opp_arg a = opp_arg_gbl((double*)nullptr, dim, typ, acc);
    a.size = dim * (int)sizeof(bool);
    a.data = (char*)data;
    return a;
}

opp_arg opp_arg_dat(opp_dat dat, int idx, opp_map map, int dim, const char* typ, opp_map p2c_map, opp_access acc,
                    bool offset) {
    opp_arg a{};
    a.argtype = OPP_ARG_DAT;
    a.dat = dat;
    a.map = map;
    a.p2c_map = p2c_map ? p2c_map->p2c_dat : nullptr;
    a.dim = dim;
    a.idx = idx;
    a.size = dat ? dat->size : 0;
    a.data = dat ? dat->data : nullptr;
    a.data_d = dat ? dat->data_d : nullptr;
    a.map_data = map ? map->map : nullptr;
    a.map_data_d = map ? map->map_d : nullptr;
    a.type = typ;
    a.acc = acc;
    a.opt = offset ? 1 : 0;
    return a;
}
opp_arg opp_arg_dat(opp_dat dat, int idx, opp_map map, opp_map p2c_map, opp_access acc, bool offset) {
    return opp_arg_dat(dat, idx, map, dat->dim, dat->type, p2c_map, acc, offset);
}
opp_arg opp_arg_dat(opp_dat dat, int idx, opp_map map, opp_access acc, bool offset) {
    return opp_arg_dat(dat, idx, map, dat->dim, dat->type, nullptr, acc, offset);
}
opp_arg opp_arg_dat(opp_dat dat, opp_map p2c_map, opp_access acc, bool offset) {
    return opp_arg_dat(dat, -1, nullptr, dat->dim, dat->type, p2c_map, acc, offset);
}
opp_arg opp_arg_dat(opp_dat dat, opp_access acc, bool offset) {
    return opp_arg_dat(dat, -1, nullptr, dat->dim, dat->type, nullptr, acc, offset);
}
opp_arg opp_arg_dat(opp_map data_map, opp_access acc, bool offset) {
    if (data_map->from->is_particle) return opp_arg_dat(data_map->p2c_dat, acc, offset);
    return opp_arg_dat(data_map, -1, nullptr, nullptr, acc, offset);
}
opp_arg opp_arg_dat(opp_map data_map, opp_map p2c_map, opp_access acc, bool offset) {
    return opp_arg_dat(data_map, -1, nullptr, p2c_map, acc, offset);
}
opp_arg opp_arg_dat(opp_map data_map, int idx, opp_map map, opp_access acc, bool offset) {
    return opp_arg_dat(data_map, idx, map, nullptr, acc, offset);
}
opp_arg opp_arg_dat(opp_map data_map, int idx, opp_map map, opp_map p2c_map, opp_access acc, bool offset) {
    opp_arg a{};
    a.argtype = OPP_ARG_MAP;
    a.map = map;
    a.dim = data_map->dim;
    a.idx = idx;
    a.size = data_map->dim * (int)sizeof(int);
    a.map_data = data_map->map;
    a.map_data_d = data_map->map_d;
    a.p2c_map = p2c_map ? p2c_map->p2c_dat : nullptr;
    a.type = "int";
    a.acc = acc;
    a.opt = offset ? 1 : 0;
    return a;
}

// --------------------------------------------------------------- particles

namespace {
// Grow every particle dat of the set to `cap` on the device (no host round trip).
void grow_particle_set(opp_set set, int cap) {
    const int old_stride = stride_of(set);
    for (opp_dat d : *set->particle_dats) {
        const int eb = elem_bytes(d);
        char* nd = dev_alloc((size_t)cap * d->size);
        char* ns = dev_alloc((size_t)cap * d->size);
        if (set->size > 0)
            check_cuda(cudaMemcpy2DAsync(nd, (size_t)cap * eb, d->data_d, (size_t)old_stride * eb, (size_t)set->size * eb,
                                         d->dim, cudaMemcpyDeviceToDevice, rt().stream),
                       "grow copy");
        if (d->is_cell_index)
            for (int c = 0; c < d->dim; c++)
                check_oppb(oppb_fill(nd + ((size_t)c * cap + set->size) * eb, cap - set->size, 4,
                                     (uint32_t)MAX_CELL_INDEX, rt().stream),
                           "fill");
        check_cuda(cudaStreamSynchronize(rt().stream), "grow sync");
        dev_free(d->data_d);
        dev_free(d->data_swap_d);
        d->data_d = nd;
        d->data_swap_d = ns;
        char* h = static_cast<char*>(std::realloc(d->data, (size_t)cap * d->size));
        if (!h) opp_abort("host realloc");
        d->data = h;
        d->version++;
    }
    set->set_capacity = cap;
}
}  // namespace

void opp_increase_particle_count(opp_set set, int insert_count) {
    // opp_increase_particle_count_core semantics (opp_increase_part_count_core.cpp:35-110).
    if (insert_count <= 0) return;
    const int new_size = set->size + insert_count;
    if (new_size > set->set_capacity) {
        const size_t cap = (size_t)set->size + (size_t)((double)insert_count * OPP_part_alloc_mult);
        if (cap > (size_t)INT32_MAX) opp_abort("particle capacity exceeds int32");
        grow_particle_set(set, std::max((int)cap, new_size));
    }
    set->size = new_size;
    set->diff = insert_count;
}

void opp_inc_part_count_with_distribution(opp_set set, int insert_count, opp_dat part_dist, bool) {
    opp_profiler->start("IncPartCountWithDistribution");
    opp_increase_particle_count(set, insert_count);
    oppb_rt::sync_host_to_device(part_dist);
    const oppb_inlet inlet{part_dist->set->size, reinterpret_cast<const int32_t*>(part_dist->data_d), nullptr,
                           nullptr};
    check_oppb(oppb_assign_faces(&inlet, reinterpret_cast<int32_t*>(set->mesh_relation_dat->data_d),
                                 set->size - set->diff, set->diff, rt().stream),
               "oppb_assign_faces");
    oppb_rt::mark_device_written(set->mesh_relation_dat);
    opp_profiler->end("IncPartCountWithDistribution");
}

void opp_reset_num_particles_to_insert(opp_set set) { set->diff = 0; }

void opp_init_particle_move(opp_set set, int, opp_arg*) {
    set->particle_remove_count = 0;
    OPP_iter_start = 0;
    OPP_iter_end = set->size;
    OPP_comm_iteration = 0;
}

bool opp_finalize_particle_move(opp_set set) {
    // opp_finalize_particle_move_core (opp_particle_organize_core.cpp:49-95), one GPU.
    oppb_move_status st{};
    check_cuda(cudaMemcpyAsync(&st, rt().status, sizeof st, cudaMemcpyDeviceToHost, rt().stream), "status");
    check_cuda(cudaStreamSynchronize(rt().stream), "status sync");
    if (st.error) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "move of set %s: %s (particle %d)", set->name, oppb_status_string(st.error),
                      st.error_index);
        opp_abort(msg);
    }
    set->particle_remove_count = st.remove_count;
    if (set->particle_remove_count <= 0) return false;
    // The organize rule of opp_finalize_particle_move_core (opp_particle_organize_core.cpp:61-92).
    const bool periodic = OPP_fill_type == OPP_Sort_Periodic || OPP_fill_type == OPP_Shuffle_Periodic;
    const bool hole_fill = OPP_fill_type == OPP_HoleFill_All ||
                           (periodic && (OPP_main_loop_iter % OPP_fill_period != 0 || OPP_comm_iteration != 0));
    const bool sort = !hole_fill && (OPP_fill_type == OPP_Sort_All || OPP_fill_type == OPP_Sort_Periodic);
    const bool shuffle = !hole_fill && (OPP_fill_type == OPP_Shuffle_All || OPP_fill_type == OPP_Shuffle_Periodic);
    if (!hole_fill && !sort && !shuffle) opp_abort("OPP_fill_type is undefined");
    std::vector<oppb_dat> dats;
    int key = -1;
    for (opp_dat d : *set->particle_dats) {
        if (d == set->mesh_relation_dat) key = (int)dats.size();
        dats.push_back(oppb_dat{d->data_d, d->data_swap_d, d->dim, elem_bytes(d)});
    }
    if (sort) {
        opp_profiler->start("Mv_sort_core");
        opp_particle_sort(set);
        opp_profiler->end("Mv_sort_core");
    } else if (shuffle) {
        // Random keys, removed particles last (oppb_shuffle); the seed follows the reference's
        // RandomFunctor seed 123 and the iteration, so each shuffle draws new keys.
        opp_profiler->start("Mv_shuffle_core");
        if (key < 0) opp_abort("opp_finalize_particle_move: set has no mesh relation");
        const int n_cells = set->cells_set ? set->cells_set->size : 0;
        const uint64_t seed = (uint64_t(123) << 32) | (uint32_t)OPP_main_loop_iter | (uint64_t(1) << 63);
        const size_t need = oppb_sort_workspace_bytes(set->size, n_cells);
        check_oppb(oppb_shuffle(set->size, n_cells, stride_of(set), (int)dats.size(), dats.data(), key, seed, nullptr,
                                oppb_rt::workspace(need), need, rt().stream),
                   "oppb_shuffle");
        for (opp_dat d : *set->particle_dats) std::swap(d->data_d, d->data_swap_d);
        opp_profiler->end("Mv_shuffle_core");
    } else {
        opp_profiler->start("Mv_holefill_core");
        const size_t need = oppb_hole_fill_workspace_bytes(set->size, set->particle_remove_count);
        check_oppb(oppb_hole_fill(set->size, set->particle_remove_count, oppb_rt::remove_bits(set), stride_of(set),
                                  (int)dats.size(), dats.data(), oppb_rt::workspace(need), need, rt().stream),
                   "oppb_hole_fill");
        opp_profiler->end("Mv_holefill_core");
    }
    for (opp_dat d : *set->particle_dats) oppb_rt::mark_device_written(d);
    set->size -= set->particle_remove_count;
    (void)key;
    return false;
}

void opp_particle_sort(opp_set set) {
    std::vector<oppb_dat> dats;
    int key = -1;
    for (opp_dat d : *set->particle_dats) {
        if (d == set->mesh_relation_dat) key = (int)dats.size();
        dats.push_back(oppb_dat{d->data_d, d->data_swap_d, d->dim, elem_bytes(d)});
    }
    if (key < 0) opp_abort("opp_particle_sort: set has no mesh relation");
    const int n_cells = set->cells_set ? set->cells_set->size : 0;
    const size_t need = oppb_sort_workspace_bytes(set->size, n_cells);
    check_oppb(oppb_sort_by_cell(set->size, n_cells, stride_of(set), (int)dats.size(), dats.data(), key, nullptr,
                                 oppb_rt::workspace(need), need, rt().stream),
               "oppb_sort_by_cell");
    for (opp_dat d : *set->particle_dats) {
        std::swap(d->data_d, d->data_swap_d);
        oppb_rt::mark_device_written(d);
    }
}

void opp_reset_dat_impl(opp_dat dat, char* val, opp_reset) {
    oppb_rt::sync_host_to_device(dat);
    const int eb = elem_bytes(dat), stride = stride_of(dat->set);
    const int n = dat->set->size;
    for (int c = 0; c < dat->dim; c++) {
        uint64_t pattern = 0;
        std::memcpy(&pattern, val + (size_t)c * eb, eb);
        check_oppb(oppb_fill(dat->data_d + (size_t)c * stride * eb, n, eb, pattern, rt().stream), "oppb_fill");
    }
    oppb_rt::mark_device_written(dat);
}

// --------------------------------------------------------------- transfers

void opp_upload_dat(opp_dat dat) {
    upload(dat, dat->set->size);
    dat->dirty_hd = NotDirty;
    dat->version++;
}

void opp_download_dat(opp_dat dat) {
    if (dat->dirty_hd == Host) {
        download(dat, dat->set->size);
        dat->dirty_hd = NotDirty;
    }
}

void opp_download_particle_set(opp_set set, bool force) {
    for (opp_dat d : *set->particle_dats) {
        if (force) d->dirty_hd = Host;
        opp_download_dat(d);
    }
}

void opp_upload_particle_set(opp_set set, bool) {
    for (opp_dat d : *set->particle_dats) opp_upload_dat(d);
}

OPP_INT* opp_get_data(opp_map map) {
    if (map->from->is_particle) return opp_get_data<OPP_INT>(map->p2c_dat);
    return map->map;
}

namespace {
// opp_print_dat_to_txtfile_core / opp_print_map_to_txtfile_core's file: files/<prefix>_<suffix>,
// the header, `rows` rows written by row(fp, i), and the marker lines after the set's own rows
// and after its exec halo (both after the last row on one GPU, where the halos are empty).
template <class Row>
void write_txt(const std::string& prefix, const char* suffix, int size, int dim, int exec, int nonexec, int rows,
               Row row) {
    const std::string file = "files/" + prefix + "_" + suffix;
    std::FILE* f = std::fopen(file.c_str(), "w");
    if (!f) {
        opp_printf("opp_print_dat_to_txtfile_core", "can't open file %s\n", file.c_str());
        std::exit(2);
    }
    std::fprintf(f, "%d %d -- %d %d\n", size, dim, exec, nonexec);
    for (int i = 0; i < rows; i++) {
        row(f, i);
        std::fprintf(f, "\n");
        if (i + 1 == size) std::fprintf(f, "import_exec_below ****************************************\n");
        if (i + 1 == size + exec) std::fprintf(f, "import_non_exec_below ****************************************\n");
    }
    std::fclose(f);
}

void print_dat_txt(opp_dat dat, const std::string& prefix, const char* suffix) {
    opp_set s = dat->set;
    const bool is_double = std::strcmp(dat->type, "double") == 0;
    write_txt(prefix, suffix, s->size, dat->dim, s->exec_size, s->nonexec_size,
              s->size + s->exec_size + s->nonexec_size, [&](std::FILE* f, int i) {
                  for (int j = 0; j < dat->dim; j++) {
                      const size_t k = (size_t)i * dat->dim + j;
                      if (is_double) {
                          // -0 is written, and left in the host copy, as +0 (as the reference does)
                          double& v = reinterpret_cast<double*>(dat->data)[k];
                          if (v == 0.0) v = 0.0;
                          std::fprintf(f, " %2.25lE", v);
                      } else {
                          std::fprintf(f, " %d", reinterpret_cast<const int*>(dat->data)[k]);
                      }
                  }
              });
}
}  // namespace

void opp_print_dat_to_txtfile(opp_dat dat, const char* prefix, const char* suffix) {
    opp_download_dat(dat);
    print_dat_txt(dat, std::string(prefix) + "_cuda", suffix);
}

void opp_print_map_to_txtfile(opp_map map, const char* prefix, const char* suffix) {
    const std::string pre = std::string(prefix) + "_cuda0_";
    if (map->from->is_particle) {  // the mesh relation dat, its device copy brought back first
        opp_download_dat(map->p2c_dat);
        print_dat_txt(map->p2c_dat, pre, suffix);
        return;
    }
    opp_set s = map->from;
    write_txt(pre, suffix, s->size, map->dim, s->exec_size, s->nonexec_size, s->size + s->exec_size,
              [&](std::FILE* f, int i) {
                  for (int j = 0; j < map->dim; j++) std::fprintf(f, " %d", map->map[(size_t)i * map->dim + j]);
              });
}

void opp_dump_dat(opp_dat dat) {
    check_cuda(cudaStreamSynchronize(rt().stream), "dump sync");
    std::fflush(stdout);
    if (dat) {
        opp_download_dat(dat);
        const bool is_double = std::strncmp("double", dat->type, 6) == 0;
        for (int i = 0; i < dat->set->size; i++) {
            for (int j = 0; j < dat->dim; j++) {
                if (!is_double) {
                    std::printf("\topp_dump_dat_core Unsupported type for dumping %s\n", dat->type);
                    std::exit(0);
                }
                std::printf("\t %+2.25lE", reinterpret_cast<const double*>(dat->data)[(size_t)i * dat->dim + j]);
            }
            std::printf("\t\n");
        }
    }
    std::fflush(stdout);
}

opp_dat opp_fetch_data(opp_dat dat) {
    if (dat->set->is_particle) {
        opp_printf("opp_fetch_data", "Error Cannot rearrange particle dats");
        opp_abort();
    }
    opp_download_dat(dat);
    return dat;
}

// One rank: no halo, so the loop runs over the set's own elements (the reference's return value
// without MPI, opp_lib/src/cuda/opp_cuda_halo.cu:318-353); the dats of the loop's arguments are
// brought current on the side that runs it: the host copy for a Device_CPU loop, the device copy
// for a Device_GPU loop.
int opp_mpi_halo_exchanges_grouped(opp_set set, int nargs, opp_arg* args, DeviceType device) {
    for (int i = 0; i < nargs; i++) {
        if (args[i].argtype != OPP_ARG_DAT || !args[i].dat) continue;
        if (device == Device_CPU) opp_download_dat(args[i].dat);
        else oppb_rt::sync_host_to_device(args[i].dat);
    }
    return set->size;
}
int opp_mpi_halo_exchanges(opp_set set, int nargs, opp_arg* args) {
    opp_mpi_halo_exchanges_grouped(set, nargs, args, Device_GPU);
    return set->size;
}
void opp_mpi_halo_exchange(opp_arg*, int) {}
void opp_mpi_halo_wait_all(int, opp_arg*) {}
void opp_mpi_force_halo_update_if_dirty(opp_set, std::vector<opp_dat> dats, DeviceType) {
    for (opp_dat d : dats) oppb_rt::sync_host_to_device(d);
}
bool is_double_indirect_reduction(opp_arg& arg) {
    return arg.argtype == OPP_ARG_DAT && arg.p2c_map != nullptr && arg.idx != -1 && arg.acc == OPP_INC;
}
void opp_init_double_indirect_reductions(int, opp_arg*) {}
void opp_exchange_double_indirect_reductions(int, opp_arg*) {}
void opp_complete_double_indirect_reductions(int, opp_arg*) {}
void opp_colour_cartesian_mesh(const int, std::vector<int>, opp_dat, const opp_dat, const int) {}
void opp_set_dirtybit_grouped(int nargs, opp_arg* args, DeviceType) {
    for (int i = 0; i < nargs; i++)
        if (args[i].argtype == OPP_ARG_DAT && args[i].dat && args[i].acc != OPP_READ)
            oppb_rt::mark_device_written(args[i].dat);
}

// ------------------------------------------------------------ B200 extras

namespace oppb_rt {

cudaStream_t stream() { return rt().stream; }

int max_hops() { return OPP_move_max_hops > 0 ? OPP_move_max_hops : 4096; }

int generation() { return g_generation; }

void* workspace(size_t bytes) {
    auto& r = rt();
    if (bytes > r.ws_bytes) {
        check_cuda(cudaStreamSynchronize(r.stream), "ws sync");
        dev_free(r.ws);
        r.ws_bytes = bytes + bytes / 4 + 256;
        r.ws = dev_alloc(r.ws_bytes);
    }
    return r.ws;
}

oppb_move_status* move_status() { return rt().status; }

uint32_t* remove_bits(opp_set set) {
    auto& e = rt().bits[set];
    const size_t words = ((size_t)stride_of(set) + 31) / 32;
    if (e.second < words) {
        check_cuda(cudaStreamSynchronize(rt().stream), "bits sync");
        dev_free(e.first);
        e.first = reinterpret_cast<uint32_t*>(dev_alloc(words * 4));
        e.second = words;
    }
    return e.first;
}

void mark_device_written(opp_dat dat) {
    dat->dirty_hd = Host;
    dat->version++;
}

void sync_host_to_device(opp_dat dat) {
    if (dat->dirty_hd == Device) {
        upload(dat, dat->set->size);
        dat->dirty_hd = NotDirty;
        dat->version++;
    }
}

const oppb_tet_mesh& tet_mesh(opp_dat c_det, opp_dat c_volume, opp_map c2c, opp_map c2n, opp_dat c_ef) {
    auto& r = rt();
    auto& M = r.mesh;
    opp_set cells = c_det ? c_det->set : c_volume ? c_volume->set : c2c ? c2c->from : c2n ? c2n->from : c_ef->set;
    if (!M.m.det) {
        const int nc = cells->size;
        size_t b[6];
        oppb_tet_mesh_bytes(nc, b);
        M.m.n_cells = nc;
        M.m.n_nodes = c2n ? c2n->to->size : 1;
        M.m.det = reinterpret_cast<double*>(dev_alloc(b[0]));
        M.m.nav = reinterpret_cast<double*>(dev_alloc(b[1]));
        M.m.c2n = reinterpret_cast<int32_t*>(dev_alloc(b[2]));
        M.m.ef = reinterpret_cast<double*>(dev_alloc(b[3]));
    }
    if (c2n && M.m.n_nodes < c2n->to->size) M.m.n_nodes = c2n->to->size;
    const double* det = nullptr;
    const double* vol = nullptr;
    const int32_t* cc = nullptr;
    const int32_t* cn = nullptr;
    const double* ef = nullptr;
    if (c_det && c_volume) {
        sync_host_to_device(c_det);
        sync_host_to_device(c_volume);
        if (M.det != c_det || M.vol != c_volume || M.det_v != c_det->version || M.vol_v != c_volume->version) {
            det = reinterpret_cast<const double*>(c_det->data_d);
            vol = reinterpret_cast<const double*>(c_volume->data_d);
            M.det = c_det, M.vol = c_volume, M.det_v = c_det->version, M.vol_v = c_volume->version;
        }
    }
    if (c2c && M.c2c != c2c) {
        cc = c2c->map_d;
        M.c2c = c2c;
    }
    if (c2n && M.c2n != c2n) {
        cn = c2n->map_d;
        M.c2n = c2n;
    }
    if (c_ef) {
        sync_host_to_device(c_ef);
        if (M.ef != c_ef || M.ef_v != c_ef->version) {
            ef = reinterpret_cast<const double*>(c_ef->data_d);
            M.ef = c_ef, M.ef_v = c_ef->version;
        }
    }
    if (det || cc || cn || ef) {
        check_oppb(oppb_tet_mesh_pack(&M.m, cells->size, det, vol, cc, cn, ef, nullptr, 0, r.invalid, r.stream),
                   "oppb_tet_mesh_pack");
        int32_t bad = 0;
        check_cuda(cudaMemcpyAsync(&bad, r.invalid, sizeof bad, cudaMemcpyDeviceToHost, r.stream), "pack check");
        check_cuda(cudaStreamSynchronize(r.stream), "pack sync");
        if (bad) opp_abort("mesh maps hold out-of-range entries");
    }
    return M.m;
}

}  // namespace oppb_rt

// ------------------------------------------------------------- direct-hop box

namespace opp {

BoundingBox::BoundingBox(const opp_dat node_pos_dat, int dim, const opp_point expansion)
    : domain_expansion(expansion), dim_(dim), node_pos_(node_pos_dat) {
    if (dim != 3 && dim != 2) opp_abort("For now, only 2D/3D BoundingBox is implemented");
    if (!node_pos_dat || node_pos_dat->dim != dim)
        opp_abort("BoundingBox: the positions must be a dat of `dim` components");
    opp_download_dat(node_pos_dat);
    const double e[3] = {expansion.x, expansion.y, expansion.z};
    double mn[3], mx[3];
    const double* p = reinterpret_cast<const double*>(node_pos_dat->data);
    const int n = node_pos_dat->set->size;
    if ((dim == 3 ? oppb_dh_bounding_box(p, n, e, mn, mx) : oppb_dh_bounding_box_2d(p, n, e, mn, mx)) != OPPB_OK)
        opp_abort("BoundingBox: no node positions");
    box_[0] = opp_point(mn[0], mn[1], mn[2]);
    box_[1] = opp_point(mx[0], mx[1], mx[2]);
}

BoundingBox::BoundingBox(int dim, opp_point min_coordinate, opp_point max_coordinate) : dim_(dim) {
    if (dim != 3 && dim != 2) opp_abort("For now, only 2D/3D BoundingBox is implemented");
    box_[0] = min_coordinate;
    box_[1] = max_coordinate;
}

}  // namespace opp
