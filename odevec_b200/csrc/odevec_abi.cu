/* C ABI of the B200 OdeVec solve path (declarations: include/odevec_b200.h).
 *
 * odevec_init    <- InitOdevec  (src/odevec.F90:94-154)
 * odevec_solve   <- SolveODE    (src/odevec.F90:158-214), device arrays
 * odevec_solve_host <- SolveODE with host arrays (copies in and out)
 * odevec_close   <- CloseOdevec (src/odevec.F90:1058-1074)
 *
 * Errors never terminate the process: API misuse returns a negative code,
 * per-cell integration failures are status codes (the reference calls
 * `stop`, src/odevec.F90:114-124, 272-287, 380-390, 585-597). */
#include <cuda.h>
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>

#include "../../include/odevec_b200.h"
#include "ov_launch.h"
#include "gen/includes_c.inc"

/* launchers, one per variant and arithmetic mode (kernels_<cid>_<mode>.cu) */
#define OV_NET(cid, TAG)                                                                       \
    namespace ov {                                                                             \
    namespace exact {                                                                          \
    cudaError_t launch_##cid(const LaunchArgs&, int, int, int, int, int, cudaStream_t);        \
    }                                                                                          \
    namespace fma {                                                                            \
    cudaError_t launch_##cid(const LaunchArgs&, int, int, int, int, int, cudaStream_t);        \
    }                                                                                          \
    }
#include "gen/registry.inc"
#undef OV_NET

/* multi-network launchers, one per compiled set and arithmetic mode
   (multi_<sid>_<mode>.cu) */
#define OV_MULTI(sid, ...)                                                                     \
    namespace ov {                                                                             \
    namespace exact {                                                                          \
    cudaError_t launch_multi_##sid(MultiArgs&, int, cudaStream_t);                             \
    }                                                                                          \
    namespace fma {                                                                            \
    cudaError_t launch_multi_##sid(MultiArgs&, int, cudaStream_t);                             \
    }                                                                                          \
    }
#include "gen/multi.inc"
#undef OV_MULTI

namespace {

struct NetEntry {
    const char* tag;
    const int* sizes;       /* neq, nnz, nrea, dense, idx_tgas, solver-state species, LUmethod */
    const double* defaults; /* nvector, dt_min */
    const double* mass;     /* species masses (g), 0 where none */
    const double* imass;    /* inverse masses (1/g) */
    ov::launch_fn exact;
    ov::launch_fn fma;
};

#define OV_NET(cid, TAG)                                                                            \
    {TAG, ov_##cid##_sizes, ov_##cid##_defaults, ov_##cid##_mass, ov_##cid##_imass, ov::exact::launch_##cid, \
     ov::fma::launch_##cid},
const NetEntry g_nets[] = {
#include "gen/registry.inc"
};
#undef OV_NET
constexpr int g_nnets = (int)(sizeof g_nets / sizeof g_nets[0]);

/* the sets of variants a multi-network kernel is compiled for */
#define OV_MULTI(sid, ...) const char* const g_multi_tags_##sid[] = {__VA_ARGS__, nullptr};
#include "gen/multi.inc"
#undef OV_MULTI
struct MultiEntry {
    const char* const* tags;
    ov::multi_fn exact;
    ov::multi_fn fma;
};
#define OV_MULTI(sid, ...) {g_multi_tags_##sid, ov::exact::launch_multi_##sid, ov::fma::launch_multi_##sid},
const MultiEntry g_multi[] = {
#include "gen/multi.inc"
    {nullptr, nullptr, nullptr}};
#undef OV_MULTI

/* tuned launch options per (variant, precision, group size, GPU model),
   generated from the autotuner's table (odevec_b200/autotune.py) */
struct TuneEntry {
    const char* tag;
    int precision, group;
    const char* device;
    int staging, jac_batch, ss_batch, max_wait;
};
#define OV_TUNE(tag, prec, grp, dev, st, jb, sb, mw) {tag, prec, grp, dev, st, jb, sb, mw},
const TuneEntry g_tune[] = {
#include "gen/tuning.inc"
    {nullptr, 0, 0, nullptr, 0, 0, 0, 0}};
#undef OV_TUNE

/* name of the current device, read once per device */
const char* current_device_name()
{
    static std::mutex mu;
    static char names[16][256];
    static bool known[16];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 16)
        return "";
    std::lock_guard<std::mutex> lock(mu);
    if (!known[dev]) {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, dev) != cudaSuccess)
            return "";
        std::snprintf(names[dev], sizeof names[dev], "%s", p.name);
        known[dev] = true;
    }
    return names[dev];
}

thread_local char g_err[512] = "";

int32_t fail(int32_t code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

/* automatic staging (the measured best on B200 without a tuning table):
   thread-local arrays, 3 blocks of 128 threads per SM for per-cell control
   up to 32 solver-state species, 2 blocks above (more registers per cell),
   2 blocks for lockstep groups.  The warp-per-cell staging (7) is slower on
   the shipped networks and is only used when asked for. */
int auto_staging(const NetEntry& e, int group_size)
{
    if (group_size != 1)
        return 1;
    return e.sizes[5] > 32 ? 1 : 3;
}

int find_net(const char* tag)
{
    if (!tag)
        return -1;
    for (int i = 0; i < g_nnets; ++i)
        if (std::strcmp(g_nets[i].tag, tag) == 0)
            return i;
    return -1;
}

}  // namespace

struct odevec_solver {
    int net;
    int64_t max_cells;
    odevec_opts opts; /* resolved */
    int device;
    unsigned long long* d_queue;
    /* staging for odevec_solve_host */
    double *d_y, *d_t, *d_dt, *d_tstop;
    uint8_t* d_mask;
    int32_t *d_status, *d_stats;
    cudaStream_t stream;
    /* FP32-LU escalation: input copies, per-cell status and retry mask */
    int64_t fb_cells;
    double *fb_y, *fb_t, *fb_dt;
    int32_t* fb_status;
    uint8_t* fb_mask;
    /* odevec_set_yield: the kernels stop starting cells while *yield != 0 */
    const int32_t* yield;
    /* visit order, longest integration span first (per-cell control):
       16-bit keys and cell indices, double-buffered for the radix sort, its
       scratch, and the order of the last solve (a continuation reuses it) */
    int64_t ord_cells;
    uint16_t* ord_keys;
    int32_t* ord_vals;
    void* ord_temp;
    size_t ord_temp_bytes;
    const int32_t* ord_cur;
};
/* d_queue words: [0] the solve's work counter, [1] cells that failed with
   FP32 factors, [2] the FP64 re-solve's work counter */
/* solves of fewer cells keep the given visit order: the order costs a
   sort, and where a persistent grid holds (nearly) every cell at once
   (19k-57k lanes resident) there is no tail to shorten */
constexpr int64_t OV_ORDER_MIN_CELLS = 32768;

namespace {
/* sort keys of the visit order: the top 16 bits of t_stop - t (a
   non-negative double's bits order as its value: sign, exponent and 4
   mantissa bits, buckets of 1/16 octave); NaN and non-positive spans 0 */
__global__ void ov_order_keys(int64_t ncells, const double* t, const double* t_stop, uint16_t* key,
                              int32_t* idx)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncells;
         c += (int64_t)gridDim.x * blockDim.x) {
        const double span = t_stop[c] - t[c];
        key[c] = span > 0.0 ? (uint16_t)((unsigned long long)__double_as_longlong(span) >> 48) : (uint16_t)0;
        idx[c] = (int32_t)c;
    }
}

/* cells whose FP32-LU solve failed get their inputs back and a retry mask;
   *nfail counts them */
/* mass fraction <-> number density (tests/primordial.f90:113-140), one
   thread per cell, species-major so every species row is a coalesced sweep */
#define OV_MASS_MAX 64
struct ov_mass_tab {
    double m[OV_MASS_MAX];
    double im[OV_MASS_MAX];
    int neq;
};

__global__ void __launch_bounds__(256) ov_convert(int64_t ncells, int direction, const double* in, double* out,
                                                  const double* rho, const ov_mass_tab tab)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += stride) {
        const double r = rho[c];
        for (int j = 0; j < tab.neq; ++j) {
            const double v = in[(int64_t)j * ncells + c];
            double o = v;
            if (tab.m[j] != 0.0)
                o = direction == OV_X2N ? r * v * tab.im[j] : v * tab.m[j] / r;
            out[(int64_t)j * ncells + c] = o;
        }
    }
}

__global__ void ov_escalate(int64_t ncells, int64_t stride, int neq, double* y, double* t, double* dt,
                            const double* y_in, const double* t_in, const double* dt_in,
                            const int32_t* status, const uint8_t* mask, uint8_t* retry,
                            unsigned long long* nfail, const unsigned long long* started)
{
    /* after a launch that yielded before starting every cell nothing is
       final yet: the pass runs after the launch that completes the solve */
    if (*started < (unsigned long long)ncells)
        return;
    /* y rows have the launch's stride, the saved inputs y_in are packed */
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncells;
         c += (int64_t)gridDim.x * blockDim.x) {
        const bool bad = status[c] != OV_OK && (!mask || mask[c]);
        retry[c] = bad ? 1 : 0;
        if (bad) {
            for (int s = 0; s < neq; ++s)
                y[(int64_t)s * stride + c] = y_in[(int64_t)s * ncells + c];
            t[c] = t_in[c];
            dt[c] = dt_in[c];
            atomicAdd(nfail, 1ull);
        }
    }
}
}  // namespace

static int32_t resolve_opts(const NetEntry& e, const odevec_opts* in, odevec_opts* out)
{
    odevec_opts o;
    if (in)
        o = *in;
    else {
        std::memset(&o, 0, sizeof o);
        o.rtol = 1e-4;
        o.atol = 1e-20;
        o.dt_min = -1.0;
    }
    if (!(o.rtol > 0.0) || !(o.atol >= 0.0))
        return fail(OV_API_EINVAL, "rtol must be > 0 and atol >= 0 (got %g, %g)", o.rtol, o.atol);
    if (o.dt_min < 0.0)
        o.dt_min = e.defaults[1];
    if (o.group_size == 0)
        o.group_size = (int)e.defaults[0] == 32 ? 32 : 1;
    if (o.group_size != 1 && o.group_size != 32)
        return fail(OV_API_EINVAL, "group_size must be 1 or 32 (got %d)", o.group_size);
    if (o.precision < OV_PREC_FP64 || o.precision > OV_PREC_FP32_LU)
        return fail(OV_API_EINVAL, "unknown precision %d", o.precision);
    if (o.max_attempts <= 0)
        o.max_attempts = 1000000;
    if (o.staging == 0 || o.jac_batch == 0 || o.ss_batch == 0 || o.max_wait == 0) {
        /* options left at 0 take the tuned values for this GPU, if any */
        const char* dev = nullptr;
        for (const TuneEntry* t = g_tune; t->tag; ++t) {
            if (t->precision != o.precision || t->group != o.group_size || std::strcmp(t->tag, e.tag) != 0)
                continue;
            if (!dev)
                dev = current_device_name();
            if (std::strcmp(t->device, dev) != 0)
                continue;
            if (o.staging == 0) o.staging = t->staging;
            if (o.jac_batch == 0) o.jac_batch = t->jac_batch;
            if (o.ss_batch == 0) o.ss_batch = t->ss_batch;
            if (o.max_wait == 0) o.max_wait = t->max_wait;
            break;
        }
    }
    if (o.jac_batch <= 0)
        o.jac_batch = 24;
    if (o.ss_batch <= 0)
        o.ss_batch = 24;
    if (o.max_wait <= 0)
        o.max_wait = o.max_wait < 0 ? 0 : 8;
    if (o.jac_batch > 32 || o.ss_batch > 32)
        return fail(OV_API_EINVAL, "jac_batch and ss_batch must be <= 32");
    if (o.staging < 0 || o.staging > 21)
        return fail(OV_API_EINVAL, "staging must be 0..21");
    if (o.block_threads < 0 || o.block_threads > 128 || o.block_threads % 32)
        return fail(OV_API_EINVAL, "block_threads must be 32, 64, 96 or 128 (0: automatic)");
    if (o.grid_blocks < 0)
        return fail(OV_API_EINVAL, "grid_blocks < 0");
    *out = o;
    return OV_API_OK;
}

extern "C" {

int32_t odevec_num_networks(void) { return g_nnets; }

const char* odevec_network_tag(int32_t i) { return (i >= 0 && i < g_nnets) ? g_nets[i].tag : nullptr; }

int32_t odevec_network_info(const char* tag, int32_t* info)
{
    const int i = find_net(tag);
    if (i < 0)
        return fail(OV_API_ENONET, "unknown network variant '%s'", tag ? tag : "(null)");
    if (!info)
        return fail(OV_API_EINVAL, "info is null");
    for (int k = 0; k < 5; ++k)
        info[k] = g_nets[i].sizes[k];
    info[5] = (int)g_nets[i].defaults[0] == 32 ? 32 : 1;
    return OV_API_OK;
}

const char* odevec_last_error(void) { return g_err; }

int32_t odevec_init(const char* network, int64_t max_cells, const odevec_opts* opts, odevec_solver** out)
{
    if (!out)
        return fail(OV_API_EINVAL, "out is null");
    *out = nullptr;
    const int ni = find_net(network);
    if (ni < 0)
        return fail(OV_API_ENONET, "unknown network variant '%s'", network ? network : "(null)");
    if (max_cells < 0)
        return fail(OV_API_EINVAL, "max_cells < 0");
    odevec_opts o;
    int32_t rc = resolve_opts(g_nets[ni], opts, &o);
    if (rc)
        return rc;
    odevec_solver* s = new (std::nothrow) odevec_solver();
    if (!s)
        return fail(OV_API_ENOMEM, "out of host memory");
    s->net = ni;
    s->max_cells = max_cells;
    s->opts = o;
    cudaError_t e = cudaGetDevice(&s->device);
    if (e == cudaSuccess)
        e = cudaMalloc(&s->d_queue, 256);
    const int neq = g_nets[ni].sizes[0];
    if (e == cudaSuccess && max_cells > 0) {
        const size_t nc = (size_t)max_cells;
        if (e == cudaSuccess) e = cudaMalloc(&s->d_y, sizeof(double) * nc * neq);
        if (e == cudaSuccess) e = cudaMalloc(&s->d_t, sizeof(double) * nc);
        if (e == cudaSuccess) e = cudaMalloc(&s->d_dt, sizeof(double) * nc);
        if (e == cudaSuccess) e = cudaMalloc(&s->d_tstop, sizeof(double) * nc);
        if (e == cudaSuccess) e = cudaMalloc(&s->d_mask, nc);
        if (e == cudaSuccess) e = cudaMalloc(&s->d_status, sizeof(int32_t) * nc);
        if (e == cudaSuccess) e = cudaMalloc(&s->d_stats, sizeof(int32_t) * nc * OV_NSTATS);
    }
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        odevec_close(s);
        return fail(e == cudaErrorMemoryAllocation ? OV_API_ENOMEM : OV_API_ECUDA, "odevec_init: %s",
                    cudaGetErrorString(e));
    }
    *out = s;
    return OV_API_OK;
}

int32_t odevec_set_options(odevec_solver* s, const odevec_opts* opts)
{
    if (!s || !opts)
        return fail(OV_API_EINVAL, "null argument");
    odevec_opts o;
    int32_t rc = resolve_opts(g_nets[s->net], opts, &o);
    if (rc)
        return rc;
    s->opts = o;
    return OV_API_OK;
}

static int32_t solve_impl(odevec_solver* s, int64_t ncells, int64_t stride, double* y, double* t,
                          double* dt, const double* t_stop, const uint8_t* mask, int32_t* status,
                          int32_t* stats, double* ws, int32_t resume, void* stream, bool cont = false);

int32_t odevec_solve(odevec_solver* s, int64_t ncells, double* y, double* t, double* dt,
                     const double* t_stop, const uint8_t* mask, int32_t* status, int32_t* stats,
                     void* stream)
{
    return solve_impl(s, ncells, ncells, y, t, dt, t_stop, mask, status, stats, nullptr, 0, stream);
}

int32_t odevec_workspace_doubles(const char* network, int64_t* per_cell)
{
    const int i = find_net(network);
    if (i < 0)
        return fail(OV_API_ENONET, "unknown network variant '%s'", network ? network : "(null)");
    if (!per_cell)
        return fail(OV_API_EINVAL, "per_cell is null");
    *per_cell = ov::ws_doubles(g_nets[i].sizes[5]);
    return OV_API_OK;
}

int32_t odevec_solve_resident(odevec_solver* s, int64_t ncells, double* y, double* t, double* dt,
                              const double* t_stop, const uint8_t* mask, int32_t* status,
                              int32_t* stats, double* workspace, int32_t resume, void* stream)
{
    if (!workspace)
        return fail(OV_API_EINVAL, "odevec_solve_resident: workspace is null");
    if (resume < 0 || resume > 2)
        return fail(OV_API_EINVAL, "odevec_solve_resident: resume must be 0, 1 or 2 (got %d)", resume);
    return solve_impl(s, ncells, ncells, y, t, dt, t_stop, mask, status, stats, workspace, resume, stream);
}

int32_t odevec_solve_range(odevec_solver* s, int64_t ncells, int64_t stride, double* y, double* t, double* dt,
                           const double* t_stop, const uint8_t* mask, int32_t* status, int32_t* stats,
                           double* workspace, int32_t resume, void* stream)
{
    if (resume < 0 || resume > 2)
        return fail(OV_API_EINVAL, "odevec_solve_range: resume must be 0, 1 or 2 (got %d)", resume);
    if (resume && !workspace)
        return fail(OV_API_EINVAL, "odevec_solve_range: resume needs a workspace");
    return solve_impl(s, ncells, stride, y, t, dt, t_stop, mask, status, stats, workspace, resume, stream);
}

int32_t odevec_set_yield(odevec_solver* s, const int32_t* flag)
{
    if (!s)
        return fail(OV_API_EINVAL, "solver is null");
    s->yield = flag;
    return OV_API_OK;
}

int32_t odevec_solve_continue(odevec_solver* s, int64_t ncells, int64_t stride, double* y, double* t, double* dt,
                              const double* t_stop, const uint8_t* mask, int32_t* status, int32_t* stats,
                              double* workspace, int32_t resume, void* stream)
{
    if (resume < 0 || resume > 2)
        return fail(OV_API_EINVAL, "odevec_solve_continue: resume must be 0, 1 or 2 (got %d)", resume);
    if (resume && !workspace)
        return fail(OV_API_EINVAL, "odevec_solve_continue: resume needs a workspace");
    return solve_impl(s, ncells, stride, y, t, dt, t_stop, mask, status, stats, workspace, resume, stream, true);
}

int32_t odevec_cells_started(odevec_solver* s, void* stream, int64_t* started)
{
    if (!s || !started)
        return fail(OV_API_EINVAL, "solver or started is null");
    unsigned long long v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, s->d_queue, sizeof v, cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess)
        return fail(OV_API_ECUDA, "odevec_cells_started: %s", cudaGetErrorString(e));
    *started = (int64_t)v;
    return OV_API_OK;
}

/* The visit order of a per-cell solve of ncells cells (device arrays t,
   t_stop): cells with the longest integration span first, computed on
   `st` into s's buffers (*order = null below OV_ORDER_MIN_CELLS cells);
   remembered as s->ord_cur for a continuation. */
static int32_t visit_order(odevec_solver* s, int64_t ncells, const double* t, const double* t_stop,
                           cudaStream_t st, const int32_t** order)
{
    *order = nullptr;
    s->ord_cur = nullptr;
    if (ncells < OV_ORDER_MIN_CELLS || ncells > (int64_t)INT32_MAX)
        return OV_API_OK;
    cudaError_t err = cudaSuccess;
    if (s->ord_cells < ncells) {
        cudaFree(s->ord_keys); cudaFree(s->ord_vals); cudaFree(s->ord_temp);
        s->ord_keys = nullptr; s->ord_vals = nullptr; s->ord_temp = nullptr;
        s->ord_cells = 0;
        s->ord_temp_bytes = 0;
        const size_t n = (size_t)ncells;
        err = cudaMalloc(&s->ord_keys, 2 * n * sizeof(uint16_t));
        if (err == cudaSuccess) err = cudaMalloc(&s->ord_vals, 2 * n * sizeof(int32_t));
        if (err == cudaSuccess) {
            cub::DoubleBuffer<uint16_t> kb(s->ord_keys, s->ord_keys + n);
            cub::DoubleBuffer<int32_t> vb(s->ord_vals, s->ord_vals + n);
            err = cub::DeviceRadixSort::SortPairsDescending(nullptr, s->ord_temp_bytes, kb, vb, (int)n, 0, 16, st);
        }
        if (err == cudaSuccess) err = cudaMalloc(&s->ord_temp, s->ord_temp_bytes);
        if (err != cudaSuccess)
            return fail(OV_API_ENOMEM, "odevec_solve: visit order buffers: %s", cudaGetErrorString(err));
        s->ord_cells = ncells;
    }
    const size_t cap = (size_t)s->ord_cells;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    ov_order_keys<<<sms * 4, 256, 0, st>>>(ncells, t, t_stop, s->ord_keys, s->ord_vals);
    err = cudaGetLastError();
    cub::DoubleBuffer<uint16_t> kb(s->ord_keys, s->ord_keys + cap);
    cub::DoubleBuffer<int32_t> vb(s->ord_vals, s->ord_vals + cap);
    size_t bytes = s->ord_temp_bytes;
    if (err == cudaSuccess)
        err = cub::DeviceRadixSort::SortPairsDescending(s->ord_temp, bytes, kb, vb, (int)ncells, 0, 16, st);
    if (err != cudaSuccess)
        return fail(OV_API_ECUDA, "odevec_solve: visit order: %s", cudaGetErrorString(err));
    s->ord_cur = vb.Current();
    *order = s->ord_cur;
    return OV_API_OK;
}

static int32_t solve_impl(odevec_solver* s, int64_t ncells, int64_t stride, double* y, double* t,
                          double* dt, const double* t_stop, const uint8_t* mask, int32_t* status,
                          int32_t* stats, double* ws, int32_t resume, void* stream, bool cont)
{
    if (!s)
        return fail(OV_API_EINVAL, "solver is null");
    if (ncells < 0)
        return fail(OV_API_EINVAL, "ncells < 0");
    if (stride < ncells)
        return fail(OV_API_EINVAL, "stride %lld < ncells %lld", (long long)stride, (long long)ncells);
    if (ncells == 0)
        return OV_API_OK;
    if (!y || !t || !dt || !t_stop)
        return fail(OV_API_EINVAL, "y, t, dt and t_stop are required");
    const odevec_opts& o = s->opts;
    if (o.group_size == 32 && ncells % 32)
        return fail(OV_API_EINVAL, "group_size 32 needs ncells divisible by 32 (got %lld)",
                    (long long)ncells);
    const NetEntry& e = g_nets[s->net];
    ov::LaunchArgs a;
    a.ncells = ncells;
    a.stride = stride;
    a.y = y;
    a.t = t;
    a.dt = dt;
    a.t_stop = t_stop;
    a.mask = mask;
    a.status = status;
    a.stats = stats;
    a.queue = s->d_queue;
    a.rtol = o.rtol;
    a.atol = o.atol;
    a.dt_min = o.dt_min;
    a.check_neg = o.check_negatives ? 1 : 0;
    a.max_attempts = o.max_attempts;
    a.jac_batch = o.jac_batch;
    a.ss_batch = o.ss_batch;
    a.max_wait = o.max_wait;
    a.fix_restart = o.fix_restart ? 1 : 0;
    a.ws = ws;
    a.resume = resume;
    a.run_if = nullptr;
    a.save_y = a.save_t = a.save_dt = nullptr;
    a.yield = s->yield;
    a.order = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    /* a continuation keeps the work counter (and the failure count) of the
       solve it continues */
    cudaError_t err = cont ? cudaSuccess : cudaMemsetAsync(s->d_queue, 0, sizeof(unsigned long long), st);
    if (err != cudaSuccess)
        return fail(OV_API_ECUDA, "odevec_solve: %s", cudaGetErrorString(err));
    /* Visit order: cells with the longest integration span first, so that
       the persistent grid's last cells are short ones (a continuation keeps
       the order of the solve it continues).  Results do not depend on it.
       Per-cell control only: a lockstep group is 32 consecutive cells.
       (Pinned host arrays read in place are then read in scattered order:
       on PRIMORDIAL that costs about what the order gains with FP32
       factors, and gains 3 % in FP64.) */
    if (cont) {
        a.order = s->ord_cur;
    } else if (o.group_size == 1) {
        const int32_t rc = visit_order(s, ncells, t, t_stop, st, &a.order);
        if (rc)
            return rc;
    } else {
        s->ord_cur = nullptr;
    }
    const int lu = o.precision == OV_PREC_FP32_LU ? 1 : 0;
    ov::launch_fn fn = o.precision == OV_PREC_FP64 ? e.exact : e.fma;
    /* automatic (options left at 0): the tuning table for this GPU, else
       auto_staging() */
    const int stage = o.staging ? o.staging : auto_staging(e, o.group_size);
    const bool escalate = lu && !o.no_escalation;
    const int neq = e.sizes[0];
    if (escalate) {
        /* FP32 factors can be too inaccurate for a badly conditioned cell
           (Newton then fails until dt < dt_min): such cells are solved again
           from their inputs with FP64 factors */
        if (cont && s->fb_cells < ncells)
            return fail(OV_API_EINVAL, "odevec_solve_continue: no solve of %lld cells to continue",
                        (long long)ncells);
        if (s->fb_cells < ncells) {
            cudaFree(s->fb_y); cudaFree(s->fb_t); cudaFree(s->fb_dt); cudaFree(s->fb_status); cudaFree(s->fb_mask);
            s->fb_y = nullptr; s->fb_t = nullptr; s->fb_dt = nullptr; s->fb_status = nullptr; s->fb_mask = nullptr;
            s->fb_cells = 0;
            const size_t n = (size_t)ncells;
            err = cudaMalloc(&s->fb_y, sizeof(double) * n * neq);
            if (err == cudaSuccess) err = cudaMalloc(&s->fb_t, sizeof(double) * n);
            if (err == cudaSuccess) err = cudaMalloc(&s->fb_dt, sizeof(double) * n);
            if (err == cudaSuccess) err = cudaMalloc(&s->fb_status, sizeof(int32_t) * n);
            if (err == cudaSuccess) err = cudaMalloc(&s->fb_mask, n);
            if (err != cudaSuccess)
                return fail(OV_API_ENOMEM, "odevec_solve: escalation buffers: %s", cudaGetErrorString(err));
            s->fb_cells = ncells;
        }
        /* the kernel saves each cell's inputs as it loads them (packed by
           ncells), so the inputs are read once, wherever they live */
        a.save_y = s->fb_y;
        a.save_t = s->fb_t;
        a.save_dt = s->fb_dt;
        err = cont ? cudaSuccess : cudaMemsetAsync(s->d_queue + 1, 0, sizeof(unsigned long long), st);
        if (err != cudaSuccess)
            return fail(OV_API_ECUDA, "odevec_solve: %s", cudaGetErrorString(err));
        if (!a.status)
            a.status = s->fb_status;
    }
    err = fn(a, o.group_size, lu, stage, o.block_threads, o.grid_blocks, st);
    if (escalate && err == cudaSuccess) {
        int blocks = 0;
        cudaDeviceGetAttribute(&blocks, cudaDevAttrMultiProcessorCount, s->device);
        ov_escalate<<<blocks * 4, 256, 0, st>>>(ncells, stride, neq, y, t, dt, s->fb_y, s->fb_t, s->fb_dt,
                                                a.status, mask, s->fb_mask, s->d_queue + 1, s->d_queue);
        err = cudaGetLastError();
        if (err == cudaSuccess) {
            ov::LaunchArgs b = a;
            b.mask = s->fb_mask;
            b.stats = nullptr;
            b.run_if = s->d_queue + 1;
            b.save_y = b.save_t = b.save_dt = nullptr;
            b.yield = nullptr; /* the re-solve runs to the end */
            b.queue = s->d_queue + 2;
            err = cudaMemsetAsync(s->d_queue + 2, 0, sizeof(unsigned long long), st);
            /* the FP64 re-solve runs rarely and only for failed cells: it
               uses the thread-local staging compiled for every variant (some
               stagings exist for FP32 factors only) */
            const int stage64 = o.group_size == 1 ? 3 : 1;
            if (err == cudaSuccess)
                err = e.fma(b, o.group_size, 0, stage64, o.block_threads, o.grid_blocks, st);
        }
    }
    if (err == cudaErrorNotSupported)
        return fail(OV_API_EUNSUPPORTED, "variant %s: group %d precision %d not compiled", e.tag,
                    o.group_size, o.precision);
    if (err != cudaSuccess)
        return fail(OV_API_ECUDA, "odevec_solve launch: %s", cudaGetErrorString(err));
    return OV_API_OK;
}

/* The device address of host array p of `bytes` bytes when it is pinned and
   mapped into the device's address space (cudaHostAlloc, or cudaHostRegister
   with mapping), so that a kernel reads and writes it in place; else null.
   Both ends are checked: an array lies inside one allocation. */
static void* mapped_host(const void* p, size_t bytes)
{
    if (!p || bytes == 0)
        return nullptr;
    cudaPointerAttributes a0, a1;
    if (cudaPointerGetAttributes(&a0, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a0.type != cudaMemoryTypeHost || !a0.devicePointer)
        return nullptr;
    const char* last = static_cast<const char*>(p) + bytes - 1;
    if (cudaPointerGetAttributes(&a1, last) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a1.type != cudaMemoryTypeHost
        || static_cast<const char*>(a1.devicePointer) != static_cast<const char*>(a0.devicePointer) + bytes - 1)
        return nullptr;
    return a0.devicePointer;
}

int32_t odevec_solve_host(odevec_solver* s, int64_t ncells, double* y, double* t, double* dt,
                          const double* t_stop, const uint8_t* mask, int32_t* status, int32_t* stats)
{
    if (!s)
        return fail(OV_API_EINVAL, "solver is null");
    if (ncells < 0)
        return fail(OV_API_EINVAL, "ncells < 0");
    if (ncells == 0)
        return OV_API_OK;
    if (ncells > s->max_cells)
        return fail(OV_API_ETOOBIG, "ncells %lld exceeds max_cells %lld given to odevec_init",
                    (long long)ncells, (long long)s->max_cells);
    if (!y || !t || !dt || !t_stop)
        return fail(OV_API_EINVAL, "y, t, dt and t_stop are required");
    const int neq = g_nets[s->net].sizes[0];
    const size_t n = (size_t)ncells;
    cudaStream_t st = s->stream;
    cudaError_t e = cudaSetDevice(s->device);
    if (e != cudaSuccess)
        return fail(OV_API_ECUDA, "odevec_solve_host: %s", cudaGetErrorString(e));
    /* An array in pinned, mapped host memory is read and written by the
       kernel in place: a cell's inputs are read when the cell is set up and
       its results written when it finishes, so those transfers overlap the
       solve.  Any other array goes through the solver's device buffer, one
       copy each way; y is contiguous [neq][ncells]. */
    const size_t yb = sizeof(double) * n * neq, vb = sizeof(double) * n;
    double* my = static_cast<double*>(mapped_host(y, yb));
    double* mt = static_cast<double*>(mapped_host(t, vb));
    double* mdt = static_cast<double*>(mapped_host(dt, vb));
    const double* mts = static_cast<const double*>(mapped_host(t_stop, vb));
    const uint8_t* mm = mask ? static_cast<const uint8_t*>(mapped_host(mask, n)) : nullptr;
    int32_t* mst = status ? static_cast<int32_t*>(mapped_host(status, sizeof(int32_t) * n)) : nullptr;
    int32_t* msa = stats ? static_cast<int32_t*>(mapped_host(stats, sizeof(int32_t) * n * OV_NSTATS)) : nullptr;
    double* ky = my ? my : s->d_y;
    double* kt = mt ? mt : s->d_t;
    double* kdt = mdt ? mdt : s->d_dt;
    const double* kts = mts ? mts : s->d_tstop;
    const uint8_t* km = mask ? (mm ? mm : s->d_mask) : nullptr;
    int32_t* kst = mst ? mst : s->d_status;
    int32_t* ksa = stats ? (msa ? msa : s->d_stats) : nullptr;
    if (!my) e = cudaMemcpyAsync(s->d_y, y, yb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !mt) e = cudaMemcpyAsync(s->d_t, t, vb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !mdt) e = cudaMemcpyAsync(s->d_dt, dt, vb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !mts) e = cudaMemcpyAsync(s->d_tstop, t_stop, vb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && mask && !mm) e = cudaMemcpyAsync(s->d_mask, mask, n, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess)
        return fail(OV_API_ECUDA, "odevec_solve_host copy-in: %s", cudaGetErrorString(e));
    int32_t rc = odevec_solve(s, ncells, ky, kt, kdt, kts, km, kst, ksa, st);
    if (rc)
        return rc;
    if (!my) e = cudaMemcpyAsync(y, s->d_y, yb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && !mt) e = cudaMemcpyAsync(t, s->d_t, vb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && !mdt) e = cudaMemcpyAsync(dt, s->d_dt, vb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && status && !mst)
        e = cudaMemcpyAsync(status, s->d_status, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && stats && !msa)
        e = cudaMemcpyAsync(stats, s->d_stats, sizeof(int32_t) * n * OV_NSTATS, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return fail(OV_API_ECUDA, "odevec_solve_host: %s", cudaGetErrorString(e));
    return OV_API_OK;
}

int32_t odevec_convert(const char* network, int64_t ncells, int32_t direction, const double* in, double* out,
                       const double* rho, void* stream)
{
    const int ni = find_net(network);
    if (ni < 0)
        return fail(OV_API_ENONET, "unknown network variant '%s'", network ? network : "(null)");
    if (ncells < 0)
        return fail(OV_API_EINVAL, "ncells < 0");
    if (direction != OV_X2N && direction != OV_N2X)
        return fail(OV_API_EINVAL, "direction must be OV_X2N or OV_N2X");
    if (ncells == 0)
        return OV_API_OK;
    if (!in || !out || !rho)
        return fail(OV_API_EINVAL, "in, out and rho are required");
    const NetEntry& e = g_nets[ni];
    const int neq = e.sizes[0];
    ov_mass_tab tab;
    if (neq > OV_MASS_MAX)
        return fail(OV_API_EUNSUPPORTED, "%s: more than %d species", e.tag, OV_MASS_MAX);
    bool any = false;
    for (int j = 0; j < neq; ++j) {
        tab.m[j] = e.mass[j];
        tab.im[j] = e.imass[j];
        any = any || e.mass[j] != 0.0;
    }
    if (!any)
        return fail(OV_API_EUNSUPPORTED, "%s has no species masses", e.tag);
    tab.neq = neq;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t want = (ncells + 255) / 256;
    const int blocks = (int)(want < (int64_t)sms * 8 ? want : (int64_t)sms * 8);
    ov_convert<<<blocks, 256, 0, (cudaStream_t)stream>>>(ncells, direction, in, out, rho, tab);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess)
        return fail(OV_API_ECUDA, "odevec_convert: %s", cudaGetErrorString(err));
    return OV_API_OK;
}

int32_t odevec_close(odevec_solver* s)
{
    if (!s)
        return OV_API_OK;
    cudaFree(s->d_queue);
    cudaFree(s->ord_keys);
    cudaFree(s->ord_vals);
    cudaFree(s->ord_temp);
    cudaFree(s->d_y);
    cudaFree(s->d_t);
    cudaFree(s->d_dt);
    cudaFree(s->d_tstop);
    cudaFree(s->d_mask);
    cudaFree(s->d_status);
    cudaFree(s->d_stats);
    cudaFree(s->fb_y);
    cudaFree(s->fb_t);
    cudaFree(s->fb_dt);
    cudaFree(s->fb_status);
    cudaFree(s->fb_mask);
    if (s->stream)
        cudaStreamDestroy(s->stream);
    delete s;
    return OV_API_OK;
}

}  // extern "C"

/* ------------------------------------------------------------------------
 * Solve without any device allocation.
 *
 * odevec_init allocates a small device work counter (and, for host arrays,
 * staging buffers) with cudaMalloc.  Some callers cannot do that: a host
 * code that hands the solver its own device arrays from inside a region
 * where device allocation is forbidden or would break its memory-pool
 * discipline (an operator-split hydro step running under a fixed memory
 * budget, or an application that owns every byte of the GPU through its own
 * allocator).  odevec_solve_noalloc serves them: it launches the same solve
 * kernel on the caller's device arrays, and takes the kernel's only scratch
 * -- the 64-bit counter from which the persistent grid hands out cells --
 * from a file-scope device array that the library image carries on every
 * GPU that loads it, until the process exits.
 * ------------------------------------------------------------------------ */
namespace {

/* OV_NOALLOC_SCRATCH_BYTES of static device memory: word 0 is the cell
   counter, the rest keeps the array on its own 256-byte line. */
static __device__ __align__(256) unsigned long long ov_noalloc_scratch[OV_NOALLOC_SCRATCH_BYTES / 8];

/* A __device__ variable has its own address in every CUDA context that
   loads the library: one per device for the runtime's primary contexts, and
   another for each context a driver-API caller creates.  A context that is
   destroyed (cudaDeviceReset, cuCtxDestroy) takes its copy with it.  The
   looked-up address is therefore cached per context, keyed by the context's
   unique ID (cuCtxGetId: never reused within a process, unlike the handle),
   so a reset or another context leads to a fresh lookup, never to a stale
   address. */
constexpr int kCacheSlots = 64;
struct ScratchSlot {
    unsigned long long ctx_id;
    unsigned long long* ptr;
};
std::mutex g_noalloc_mutex;
ScratchSlot g_noalloc_cache[kCacheSlots] = {};
int g_noalloc_next = 0;
typedef CUresult (*ctx_get_current_fn)(CUcontext*);
typedef CUresult (*ctx_get_id_fn)(CUcontext, unsigned long long*);
ctx_get_current_fn g_ctx_get_current = nullptr;
ctx_get_id_fn g_ctx_get_id = nullptr;

/* ID of the current context (the runtime's primary context of the current
   device is made current first if the thread has none). */
int32_t current_context_id(unsigned long long* id)
{
    if (!g_ctx_get_current || !g_ctx_get_id) {
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
        cudaError_t e1 = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1);
        cudaError_t e2 = cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2);
        if (e1 != cudaSuccess || e2 != cudaSuccess || q1 != cudaDriverEntryPointSuccess ||
            q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
            return fail(OV_API_ECUDA, "odevec_solve_noalloc: driver entry points cuCtxGetCurrent/cuCtxGetId "
                        "unavailable (%s)", cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
        g_ctx_get_current = reinterpret_cast<ctx_get_current_fn>(f1);
        g_ctx_get_id = reinterpret_cast<ctx_get_id_fn>(f2);
    }
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS)
        return fail(OV_API_ECUDA, "odevec_solve_noalloc: cuCtxGetCurrent failed");
    if (!ctx) {
        /* no context yet on this thread: cudaSetDevice makes the runtime's
           primary context of the current device current */
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess)
            e = cudaSetDevice(dev);
        if (e != cudaSuccess)
            return fail(OV_API_ECUDA, "odevec_solve_noalloc: %s", cudaGetErrorString(e));
        if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx)
            return fail(OV_API_ECUDA, "odevec_solve_noalloc: no current CUDA context");
    }
    if (g_ctx_get_id(ctx, id) != CUDA_SUCCESS)
        return fail(OV_API_ECUDA, "odevec_solve_noalloc: cuCtxGetId failed");
    return OV_API_OK;
}

/* Device address of the static scratch in the current context.  In host
   code the name ov_noalloc_scratch is only a handle, so the address is
   looked up with cudaGetSymbolAddress once per context and cached. */
int32_t noalloc_scratch(unsigned long long** out)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    unsigned long long id = 0;
    int32_t rc = current_context_id(&id);
    if (rc)
        return rc;
    for (int i = 0; i < kCacheSlots; ++i) {
        if (g_noalloc_cache[i].ptr && g_noalloc_cache[i].ctx_id == id) {
            *out = g_noalloc_cache[i].ptr;
            return OV_API_OK;
        }
    }
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, ov_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return fail(OV_API_ECUDA, "odevec_solve_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    /* slots of destroyed contexts are never matched again (IDs are not
       reused); they are overwritten in turn once all slots are taken */
    g_noalloc_cache[g_noalloc_next] = ScratchSlot{id, static_cast<unsigned long long*>(p)};
    g_noalloc_next = (g_noalloc_next + 1) % kCacheSlots;
    *out = static_cast<unsigned long long*>(p);
    return OV_API_OK;
}

}  // namespace

extern "C" int32_t odevec_solve_noalloc(const char* network, const odevec_opts* opts, int64_t ncells,
                                        double* y, double* t, double* dt, const double* t_stop,
                                        const uint8_t* mask, int32_t* status, int32_t* stats,
                                        void* stream)
{
    const int ni = find_net(network);
    if (ni < 0)
        return fail(OV_API_ENONET, "unknown network variant '%s'", network ? network : "(null)");
    if (ncells < 0)
        return fail(OV_API_EINVAL, "ncells < 0");
    if (ncells > OV_NOALLOC_MAX_CELLS)
        return fail(OV_API_ETOOBIG, "odevec_solve_noalloc: %lld cells exceed the maximum of %lld",
                    (long long)ncells, (long long)OV_NOALLOC_MAX_CELLS);
    if (ncells == 0)
        return OV_API_OK;
    if (!y || !t || !dt || !t_stop)
        return fail(OV_API_EINVAL, "y, t, dt and t_stop are required");
    odevec_opts o;
    int32_t rc = resolve_opts(g_nets[ni], opts, &o);
    if (rc)
        return rc;
    if (o.group_size == 32 && ncells % 32)
        return fail(OV_API_EINVAL, "group_size 32 needs ncells divisible by 32 (got %lld)",
                    (long long)ncells);
    unsigned long long* counter = nullptr;
    rc = noalloc_scratch(&counter);
    if (rc)
        return rc;
    cudaStream_t st = (cudaStream_t)stream;
    /* the scratch keeps the previous call's count: the counter must start at 0 */
    cudaError_t err = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (err != cudaSuccess)
        return fail(OV_API_ECUDA, "odevec_solve_noalloc: %s", cudaGetErrorString(err));
    ov::LaunchArgs a;
    a.ncells = ncells;
    a.stride = ncells;
    a.y = y;
    a.t = t;
    a.dt = dt;
    a.t_stop = t_stop;
    a.mask = mask;
    a.status = status;
    a.stats = stats;
    a.queue = counter;
    a.rtol = o.rtol;
    a.atol = o.atol;
    a.dt_min = o.dt_min;
    a.check_neg = o.check_negatives ? 1 : 0;
    a.max_attempts = o.max_attempts;
    a.jac_batch = o.jac_batch;
    a.ss_batch = o.ss_batch;
    a.max_wait = o.max_wait;
    a.fix_restart = o.fix_restart ? 1 : 0;
    a.ws = nullptr;
    a.resume = 0;
    a.run_if = nullptr;
    a.save_y = a.save_t = a.save_dt = nullptr;
    a.yield = nullptr;
    a.order = nullptr;
    const NetEntry& e = g_nets[ni];
    const int lu = o.precision == OV_PREC_FP32_LU ? 1 : 0;
    ov::launch_fn fn = o.precision == OV_PREC_FP64 ? e.exact : e.fma;
    const int stage = o.staging ? o.staging : auto_staging(e, o.group_size);
    err = fn(a, o.group_size, lu, stage, o.block_threads, o.grid_blocks, st);
    if (err == cudaErrorNotSupported)
        return fail(OV_API_EUNSUPPORTED, "variant %s: group %d precision %d not compiled", e.tag,
                    o.group_size, o.precision);
    if (err != cudaSuccess)
        return fail(OV_API_ECUDA, "odevec_solve_noalloc launch: %s", cudaGetErrorString(err));
    return OV_API_OK;
}

/* ------------------------------------------------------------------------
 * Several networks in one launch.
 * ------------------------------------------------------------------------ */
extern "C" int32_t odevec_solve_many(const odevec_job* jobs, int32_t njobs, void* stream)
{
    if (!jobs || njobs < 1 || njobs > OV_MULTI_MAX_JOBS)
        return fail(OV_API_EINVAL, "odevec_solve_many: 1..%d jobs (got %d)", OV_MULTI_MAX_JOBS, njobs);
    int prec = -1;
    int live[OV_MULTI_MAX_JOBS];
    int nlive = 0;
    for (int j = 0; j < njobs; ++j) {
        const odevec_job& J = jobs[j];
        if (!J.solver)
            return fail(OV_API_EINVAL, "odevec_solve_many: job %d has no solver", j);
        if (J.ncells < 0)
            return fail(OV_API_EINVAL, "odevec_solve_many: job %d: ncells < 0", j);
        for (int i = 0; i < j; ++i)
            if (jobs[i].solver == J.solver)
                return fail(OV_API_EINVAL, "odevec_solve_many: jobs %d and %d share a solver", i, j);
        const odevec_opts& o = J.solver->opts;
        if (o.group_size != 1)
            return fail(OV_API_EUNSUPPORTED, "odevec_solve_many: job %d: group_size %d (per-cell control only)",
                        j, o.group_size);
        if (prec >= 0 && o.precision != prec)
            return fail(OV_API_EINVAL, "odevec_solve_many: jobs of different precision forms");
        prec = o.precision;
        if (J.ncells == 0)
            continue;
        if (!J.y || !J.t || !J.dt || !J.t_stop)
            return fail(OV_API_EINVAL, "odevec_solve_many: job %d: y, t, dt and t_stop are required", j);
        if (J.resume && !J.workspace)
            return fail(OV_API_EINVAL, "odevec_solve_many: job %d: resume needs a workspace", j);
        if (J.resume < 0 || J.resume > 2)
            return fail(OV_API_EINVAL, "odevec_solve_many: job %d: resume must be 0, 1 or 2", j);
        live[nlive++] = j;
    }
    if (nlive == 0)
        return OV_API_OK;
    /* a compiled set that holds every job's network */
    const MultiEntry* m = g_multi;
    int idx[OV_MULTI_MAX_JOBS];
    for (; m->tags; ++m) {
        bool all = true;
        for (int q = 0; q < nlive && all; ++q) {
            const char* tag = g_nets[jobs[live[q]].solver->net].tag;
            idx[q] = -1;
            for (int k = 0; m->tags[k]; ++k)
                if (std::strcmp(m->tags[k], tag) == 0)
                    idx[q] = k;
            all = idx[q] >= 0;
        }
        if (all)
            break;
    }
    if (!m->tags)
        return fail(OV_API_EUNSUPPORTED, "odevec_solve_many: no multi-network kernel compiled for this set of "
                    "networks (see odevec_b200/build.py MULTI_SETS)");
    cudaStream_t st = (cudaStream_t)stream;
    ov::MultiArgs P;
    std::memset(&P, 0, sizeof P);
    P.njobs = nlive;
    for (int q = 0; q < nlive; ++q) {
        const odevec_job& J = jobs[live[q]];
        const odevec_opts& o = J.solver->opts;
        ov::LaunchArgs& a = P.job[q];
        a.ncells = J.ncells;
        a.stride = J.ncells;
        a.y = J.y;
        a.t = J.t;
        a.dt = J.dt;
        a.t_stop = J.t_stop;
        a.mask = J.mask;
        a.status = J.status;
        a.stats = J.stats;
        a.queue = J.solver->d_queue;
        a.rtol = o.rtol;
        a.atol = o.atol;
        a.dt_min = o.dt_min;
        a.check_neg = o.check_negatives ? 1 : 0;
        a.max_attempts = o.max_attempts;
        a.jac_batch = o.jac_batch;
        a.ss_batch = o.ss_batch;
        a.max_wait = o.max_wait;
        a.fix_restart = o.fix_restart ? 1 : 0;
        a.ws = J.workspace;
        a.resume = J.resume;
        a.run_if = nullptr;
        P.net[q] = idx[q];
        cudaError_t err = cudaMemsetAsync(J.solver->d_queue, 0, sizeof(unsigned long long), st);
        if (err != cudaSuccess)
            return fail(OV_API_ECUDA, "odevec_solve_many: %s", cudaGetErrorString(err));
        /* each job's cells longest span first, as odevec_solve visits them */
        const int32_t rc = visit_order(J.solver, J.ncells, J.t, J.t_stop, st, &a.order);
        if (rc)
            return rc;
    }
    const int lu = prec == OV_PREC_FP32_LU ? 1 : 0;
    ov::multi_fn fn = prec == OV_PREC_FP64 ? m->exact : m->fma;
    cudaError_t err = fn(P, lu, st);
    if (err == cudaErrorNotSupported)
        return fail(OV_API_EUNSUPPORTED, "odevec_solve_many: precision %d not compiled", prec);
    if (err != cudaSuccess)
        return fail(OV_API_ECUDA, "odevec_solve_many launch: %s", cudaGetErrorString(err));
    return OV_API_OK;
}
