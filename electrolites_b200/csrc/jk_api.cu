// Plan construction, build engine and C ABI of the B200 J/K engine
// (declared in include/jk_b200.h).
//
// A build is a list of items, one per plan (molecule) with its densities and
// outputs.  jk_build is a list of one; jk_batch_build is a list of hundreds.
// Either way the build is the same stream of launches: one density pass over
// all items (symmetrised / transposed densities), one screening-table pass,
// then per angular-momentum class one persistent kernel over the task rows
// of every item, and one J/K assembly pass.  Every per-item pointer and size
// the kernels read comes from one descriptor blob uploaded per build (and
// skipped when it is unchanged), so a batch's launch stream can be captured
// once in a CUDA graph and replayed for new density values.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/jk_b200.h"
#include "jk_device.cuh"
#include "jk_launch.h"
#include "jk_prep.cuh"
#include "generated/class_table.inc"
#include "generated/rys_table_data.inc"

#include <cub/cub.cuh>

#define NPAIR_CLASSES 10          // (la, lb), la >= lb, l <= 3
#define PLAN_DM_MARGIN 13.815511  // log(1e6): pairs kept for |D| up to 1e6

static thread_local std::string g_err;

static int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

#define CK(call)                                                                   \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess)                                                     \
            return fail(JK_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

#define RC(call)                  \
    do {                          \
        const int r_ = (call);    \
        if (r_ != JK_OK) return r_; \
    } while (0)

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

static size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }
static int ncart(int l) { return (l + 1) * (l + 2) / 2; }
static int pair_class(int la, int lb) { return la * (la + 1) / 2 + lb; }

static double common_fac(int l)
{
    if (l == 0) return 0.282094791773878143;
    if (l == 1) return 0.488602511902919921;
    return 1.0;
}

// the class units keep per-kernel launch state (shared-memory opt-in,
// occupancy); builds from several host threads take turns there
static std::mutex g_launch_mutex;

// ---------------------------------------------------------------------------
// Rys tables: one copy per device, shared by every plan, kept until exit
// ---------------------------------------------------------------------------
static std::mutex g_rys_mutex;
static double *g_rys[JK_MAX_DEVICES];
static float *g_rys32[JK_MAX_DEVICES];

static int rys_tables(int device, const double **rys, const float **rys32)
{
    if (device < 0 || device >= JK_MAX_DEVICES) return fail(JK_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_rys_mutex);
    if (!g_rys[device]) {
        std::vector<double> h(RYS_TOTAL);
        std::memcpy(h.data(), rys_table_host, sizeof(rys_table_host));
        std::vector<float> h32(RYS32_TOTAL);
        std::memcpy(h32.data(), rys_table32_host, sizeof(rys_table32_host));
        for (int n = 0; n < RYS_NMAX; ++n)
            for (int k = 0; k < RYS_NMAX; ++k) {
                h[RYS_LARGEX_OFF + n * RYS_NMAX + k] = rys_largex_r_host[n][k];
                h[RYS_LARGEX_OFF + RYS_NMAX * RYS_NMAX + n * RYS_NMAX + k] = rys_largex_w_host[n][k];
                h32[RYS32_LARGEX_OFF + n * RYS_NMAX + k] = (float)rys_largex_r_host[n][k];
                h32[RYS32_LARGEX_OFF + RYS_NMAX * RYS_NMAX + n * RYS_NMAX + k] =
                    (float)rys_largex_w_host[n][k];
            }
        double *d = nullptr;
        float *d32 = nullptr;
        CK(cudaMalloc(&d, h.size() * sizeof(double)));
        CK(cudaMalloc(&d32, h32.size() * sizeof(float)));
        CK(cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d32, h32.data(), h32.size() * sizeof(float), cudaMemcpyHostToDevice));
        g_rys[device] = d;
        g_rys32[device] = d32;
    }
    *rys = g_rys[device];
    *rys32 = g_rys32[device];
    return JK_OK;
}

// ---------------------------------------------------------------------------
// Engine: the device state of builds -- task rows, counters, the
// descriptor blob, the workspace and the per-class tuning.  A plan owns one
// for its own builds; a batch owns one for builds over many plans.
// ---------------------------------------------------------------------------
struct ClassTune {
    int tasks_per_sm;    // tasks per SM the task size aims at
    int blocks_per_sm;   // cap on resident blocks per SM (0: occupancy limit)
    int fp32;            // mixed builds may run this class's low-bound quartets in FP32
    int jmd;             // J-only builds take the McMurchie-Davidson kernel
};

// Class kernels run on this many streams: a persistent class kernel ends
// with a tail in which the warps that have no task left idle until the last
// task of the class finishes; on two streams the next class fills those SMs.
#define JK_CLASS_STREAMS 2

struct Engine {
    int device = 0, num_sms = 148;
    // nuclear-gradient build (grad != null): its output, zeroed at launch
    double *grad = nullptr;
    size_t grad_bytes = 0;
    double grad_wj = 0., grad_wk = 0.;
    const int *grad_atom = nullptr;
    // per class stream: 4 x max_rows ints (candidates, chunks, chunk prefix,
    // candidate prefix) and CUB scratch of cub_stride bytes
    int *d_rows = nullptr;
    long long max_rows = 0;
    void *d_cub = nullptr;
    size_t cub_bytes = 0, cub_stride = 0;
    cudaStream_t side[JK_CLASS_STREAMS - 1] = {};   // class streams besides the build's
    cudaEvent_t ev_fork = nullptr;
    cudaEvent_t ev_join[JK_CLASS_STREAMS - 1] = {};
    int *d_chunk = nullptr;         // task size per class
    int *d_counters = nullptr;      // task counter per class launch
    int counter_cap = 0;
    unsigned long long *d_nq = nullptr;   // quartets, primitive quartets, FP32 quartets per class
    int *d_error = nullptr;         // {code, item}
    char *h_blob = nullptr;         // pinned staging copy of the descriptors
    char *d_blob = nullptr;
    size_t blob_cap = 0;
    std::vector<char> blob;         // descriptors of the build being prepared
    std::vector<char> blob_dev;     // descriptors on the device
    cudaEvent_t blob_ev = nullptr;  // after the last descriptor upload
    cudaEvent_t done_ev = nullptr;  // at the end of the last build
    bool blob_ev_rec = false, done_ev_rec = false;
    cudaStream_t done_stream = nullptr;
    char *d_ws = nullptr;
    size_t ws_size = 0;
    unsigned alloc_gen = 0;         // bumped whenever a buffer moves
    ClassTune tune[JK_NCLASSES];
    unsigned tune_gen = 0;
    int shard_rank = 0, shard_size = 1;
    // operator of the prepared build: sum_t op_coef[t] * (1/r, or
    // erf(omega_t r)/r with op_inv_om2[t] = 1/omega_t^2)
    int nterm = 1;
    double op_coef[2] = {1.0, 0.0}, op_inv_om2[2] = {0.0, 0.0};
    // J engine of the prepared build (one plan, J only)
    int jx = 0;
    bool jx_jonly = false;          // the J engine's build has no K
    // McMurchie-Davidson J may serve its classes: a J-only build of one plan,
    // the Coulomb operator, at most JK_MD_DENS densities
    bool md_ok = false;
    bool jx_reg = true;             // J/K builds: register-form classes too
    double *jx_dens = nullptr, *jx_acc = nullptr;
    const jk_plan *jx_plan = nullptr;
    const double *jx_ds = nullptr;
    double *jx_Jh = nullptr;
    int jx_nj = 0;
    bool timing = false;
    int timing_mode = 0;            // 1: serialised on one stream, 2: on the class streams
    std::vector<cudaEvent_t> ev;    // 2 per class
    std::vector<char> ev_used;
    int launches = 0;
    cudaStream_t last_stream = nullptr;
    const double *rys = nullptr;
    const float *rys32 = nullptr;
    // layout of the prepared build
    int nitems = 0;
    int mixed = 0;                  // the build has a mixed-precision threshold
    int cls_view0[JK_NCLASSES], cls_nview[JK_NCLASSES], cls_rows[JK_NCLASSES],
        cls_maxprim[JK_NCLASSES];
    int cls_nlaunch[JK_NCLASSES], cls_cnt0[JK_NCLASSES];   // launches per class, first counter
    int ncounters = 0;
    size_t off_views = 0, off_row0 = 0, off_pre = 0, off_post = 0, off_cond = 0, off_pair = 0;
    int npre = 0, npost = 0, npair = 0;
    long long pre_tiles = 0, post_tiles = 0, cond_blocks = 0, pair_blocks = 0;
    char *ws = nullptr;             // workspace of the prepared build
    size_t acc_bytes = 0;           // accumulators at its start (cleared per build)
};

struct jk_plan {
    int device = 0;
    int nbas_user = 0, nbas = 0, nao = 0;
    bool expanded = false;          // a general contraction was split
    std::vector<int> sh_l, sh_ao, sh_user, sh_atom;
    int natm = 0;
    double tol = 1e-13;
    float log_tol = 0.f;
    // screening threshold of the builds: the plan's own or a looser one
    // (jk_plan_set_tol), never tighter than the pair lists were made for
    double build_tol = 1e-13;
    float build_log_tol = 0.f;
    float q_max = -INFINITY, q_drop_max = -INFINITY;
    long long npairs = 0;
    long long max_rows = 0;         // largest bra-class pairs x ket-class sub-lists
    size_t table_bytes = 0;         // device memory of the plan's tables
    int pc_off[NPAIR_CLASSES + 1] = {0};
    int pc_maxprim[NPAIR_CLASSES] = {0};
    std::vector<float> q_full;      // nbas x nbas (expanded numbering)
    // device tables
    ShellDev *d_shells = nullptr;
    double *d_basis = nullptr;
    double *d_prim = nullptr;
    double *d_prim_soa = nullptr;   // field-major copy in ket order
    float *d_prim32 = nullptr;      // FP32 copies of the records (mixed form)
    PairRec *d_pairs = nullptr;
    int *d_sh_ao = nullptr, *d_sh_nf = nullptr, *d_sh_atom = nullptr;
    // ket sub-lists (equal primitive-pair count) per pair class
    std::vector<int2> subs;
    int sub_off[NPAIR_CLASSES + 1] = {0};
    int2 *d_subs = nullptr;
    double *d_io = nullptr;         // device buffers of jk_build_host
    size_t io_size = 0;
    long long nx_total = 0;         // x-space elements per density (J engine)
    bool jengine = true;            // J-only builds through the J engine
    Engine eng;                     // the plan's own builds
};

struct jk_batch {
    Engine eng;
    cudaStream_t cap_stream = nullptr;   // capture stream of the graph
    cudaGraphExec_t gexec = nullptr;
    std::vector<char> graph_blob;
    unsigned graph_alloc_gen = 0, graph_tune_gen = 0;
    int graph_spec[4] = {0, 0, 0, 0};
    double graph_mixed = 0;
    int graph_launches = 0;
    bool warmed = false;            // one build ran outside a capture
    int last_replayed = 0, last_captured = 0;
};

// ---------------------------------------------------------------------------
// engine allocation
// ---------------------------------------------------------------------------
static void engine_defaults(Engine &E)
{
    for (int c = 0; c < JK_NCLASSES; ++c) {
        E.tune[c].tasks_per_sm = jk_class_table[c].form == 0 ? 64 : 16;
        E.tune[c].blocks_per_sm = 0;
        E.tune[c].fp32 = jk_class_table[c].fp32_default;
        E.tune[c].jmd = jk_class_table[c].md_default;
    }
}

static int engine_init(Engine &E, int device)
{
    E.device = device;
    engine_defaults(E);
    CK(cudaDeviceGetAttribute(&E.num_sms, cudaDevAttrMultiProcessorCount, device));
    RC(rys_tables(device, &E.rys, &E.rys32));
    CK(cudaMalloc(&E.d_chunk, JK_NCLASSES * sizeof(int)));
    CK(cudaMalloc(&E.d_counters, JK_NCLASSES * sizeof(int)));
    E.counter_cap = JK_NCLASSES;
    CK(cudaMalloc(&E.d_nq, 3 * JK_NCLASSES * sizeof(unsigned long long)));
    CK(cudaMemset(E.d_nq, 0, 3 * JK_NCLASSES * sizeof(unsigned long long)));
    CK(cudaMalloc(&E.d_error, 2 * sizeof(int)));
    CK(cudaMemset(E.d_error, 0, 2 * sizeof(int)));
    CK(cudaEventCreateWithFlags(&E.blob_ev, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&E.done_ev, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&E.ev_fork, cudaEventDisableTiming));
    for (int s = 0; s < JK_CLASS_STREAMS - 1; ++s) {
        CK(cudaStreamCreateWithFlags(&E.side[s], cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&E.ev_join[s], cudaEventDisableTiming));
    }
    return JK_OK;
}

static void engine_free(Engine &E)
{
    cudaFree(E.d_rows);
    cudaFree(E.d_cub);
    cudaFree(E.d_chunk);
    cudaFree(E.d_counters);
    cudaFree(E.d_nq);
    cudaFree(E.d_error);
    cudaFree(E.d_blob);
    cudaFree(E.d_ws);
    if (E.h_blob) cudaFreeHost(E.h_blob);
    if (E.blob_ev) cudaEventDestroy(E.blob_ev);
    if (E.done_ev) cudaEventDestroy(E.done_ev);
    if (E.ev_fork) cudaEventDestroy(E.ev_fork);
    for (int s = 0; s < JK_CLASS_STREAMS - 1; ++s) {
        if (E.side[s]) cudaStreamDestroy(E.side[s]);
        if (E.ev_join[s]) cudaEventDestroy(E.ev_join[s]);
    }
    for (auto &e : E.ev) cudaEventDestroy(e);
    E = Engine();
}

// wait until the device no longer uses the engine's buffers
static int engine_idle(Engine &E)
{
    if (E.done_ev_rec) CK(cudaEventSynchronize(E.done_ev));
    if (E.blob_ev_rec) CK(cudaEventSynchronize(E.blob_ev));
    return JK_OK;
}

static int engine_reserve_rows(Engine &E, long long rows, bool no_alloc, const char *who)
{
    if (rows <= E.max_rows) return JK_OK;
    if (no_alloc) return fail(JK_ERR_SCRATCH, std::string(who) + ": task rows beyond the plan's reservation");
    RC(engine_idle(E));
    cudaFree(E.d_rows);
    cudaFree(E.d_cub);
    E.d_rows = nullptr;
    E.d_cub = nullptr;
    E.max_rows = 0;
    E.alloc_gen++;
    size_t cub = 0;
    CK(cub::DeviceScan::InclusiveSum(nullptr, cub, (int *)nullptr, (int *)nullptr, (int)rows));
    const size_t stride = align256(std::max<size_t>(16, cub));
    if (cudaMalloc(&E.d_rows, JK_CLASS_STREAMS * 4 * (size_t)rows * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&E.d_cub, JK_CLASS_STREAMS * stride) != cudaSuccess) {
        cudaGetLastError();
        return fail(JK_ERR_NOMEM, std::string(who) + ": cannot allocate the task rows");
    }
    E.cub_bytes = cub;
    E.cub_stride = stride;
    E.max_rows = rows;
    return JK_OK;
}

static int engine_reserve_blob(Engine &E, size_t bytes, bool no_alloc, const char *who)
{
    if (bytes <= E.blob_cap) return JK_OK;
    if (no_alloc) return fail(JK_ERR_SCRATCH, std::string(who) + ": descriptors beyond the plan's reservation");
    RC(engine_idle(E));
    cudaFree(E.d_blob);
    if (E.h_blob) cudaFreeHost(E.h_blob);
    E.d_blob = nullptr;
    E.h_blob = nullptr;
    E.blob_cap = 0;
    E.blob_dev.clear();
    E.blob_ev_rec = false;
    E.alloc_gen++;
    const size_t cap = align256(bytes + bytes / 4);
    if (cudaMalloc(&E.d_blob, cap) != cudaSuccess || cudaMallocHost(&E.h_blob, cap) != cudaSuccess) {
        cudaGetLastError();
        return fail(JK_ERR_NOMEM, std::string(who) + ": cannot allocate the build descriptors");
    }
    E.blob_cap = cap;
    return JK_OK;
}

// bytes of a descriptor blob
static size_t blob_bytes(size_t nviews, size_t npre, size_t npost, size_t ncond)
{
    return align256(nviews * sizeof(PlanView)) + align256(nviews * sizeof(int)) +
           align256(npre * sizeof(TileOp)) + align256(npost * sizeof(TileOp)) +
           align256(ncond * sizeof(CondItem));
}

// ---------------------------------------------------------------------------
// build preparation (host) and launch stream (device)
// ---------------------------------------------------------------------------
struct Item {
    jk_plan *p;
    const double *dm;
    int n_dm;
    double *vj, *vk;
    // derived
    int n_k = 0, n_j = 0, n_ka = 0;
    bool need_t = false;
    double *Kh = nullptr, *Jh = nullptr, *dsJ = nullptr, *DT = nullptr;
    double2 *dmK2 = nullptr;        // K densities interleaved in pairs
    int n_kp = 0;                   // pairs of them (0: not interleaved)
    float *dmc = nullptr, *dm_max = nullptr;
};

// The operator is sum_t coef[t] * op(omega[t]) over nterm (1 or 2) terms,
// op(0) = 1/r and op(w > 0) = erf(w r)/r.
struct Spec {
    int hermi, with_j, with_k;
    double mixed_threshold;
    int nterm;
    double coef[2];
    double omega[2];
    // nuclear gradient instead of J/K: weights of W (see jk_grad.cuh) and
    // the output, natm x 3 (device)
    int grad = 0;
    double grad_wj = 0., grad_wk = 0.;
    double *grad_out = nullptr;
};

static Spec coulomb_spec(int hermi, int with_j, int with_k, double mixed_threshold)
{
    Spec s;
    s.hermi = hermi;
    s.with_j = with_j;
    s.with_k = with_k;
    s.mixed_threshold = mixed_threshold;
    s.nterm = 1;
    s.coef[0] = 1.0;
    s.coef[1] = 0.0;
    s.omega[0] = s.omega[1] = 0.0;
    return s;
}

static int check_spec(const Spec &s, const char *who)
{
    if (s.hermi < 0 || s.hermi > 2)
        return fail(JK_ERR_ARG, std::string(who) + ": hermi must be 0, 1 or 2");
    if (s.nterm < 1 || s.nterm > 2)
        return fail(JK_ERR_ARG, std::string(who) + ": the operator takes 1 or 2 terms");
    for (int t = 0; t < s.nterm; ++t) {
        if (!(s.omega[t] >= 0) || !std::isfinite(s.omega[t]))
            return fail(JK_ERR_ARG, std::string(who) + ": omega must be finite and >= 0 (short "
                                                        "range: full minus long range)");
        if (!std::isfinite(s.coef[t]))
            return fail(JK_ERR_ARG, std::string(who) + ": operator coefficients must be finite");
    }
    return JK_OK;
}

template <class T>
static void put(std::vector<char> &blob, size_t off, const std::vector<T> &v)
{
    if (!v.empty()) std::memcpy(blob.data() + off, v.data(), v.size() * sizeof(T));
}

// Lays out the workspace and the descriptors of a build over `items`.
// ws_ext: a caller-owned workspace of ws_ext_size bytes instead of the
// engine's; no_alloc: fail instead of growing any engine buffer.
static int engine_prepare(Engine &E, std::vector<Item> &items, const Spec &s, char *ws_ext,
                          size_t ws_ext_size, bool no_alloc, const char *who)
{
    RC(check_spec(s, who));
    const int n = (int)items.size();
    if (n <= 0) return fail(JK_ERR_ARG, std::string(who) + ": no items");
    // ---- workspace: accumulators of every item, then per-item buffers ----
    // (the library's static scratch of jk_build_noalloc holds no pair copies)
    const bool pair_k = ws_ext == nullptr;
    // J engine: J of a one-plan, one-operator build outside the static
    // scratch (with K: the quartets kept for J alone)
    const bool jx = n == 1 && items[0].p && items[0].p->jengine && s.with_j && s.hermi != 2 &&
                    s.nterm == 1 && ws_ext == nullptr && !s.grad;
    size_t acc = 0, need = 0;
    for (int i = 0; i < n; ++i) {
        Item &it = items[i];
        if (!it.p) return fail(JK_ERR_ARG, std::string(who) + ": plan is NULL");
        if (it.p->device != E.device)
            return fail(JK_ERR_ARG, std::string(who) + ": plan " + std::to_string(i) +
                                        " lives on another device");
        if (it.n_dm <= 0 || !it.dm) return fail(JK_ERR_ARG, std::string(who) + ": no densities");
        if (!s.grad && ((s.with_j && !it.vj) || (s.with_k && !it.vk)))
            return fail(JK_ERR_ARG, std::string(who) + ": output is NULL");
        const size_t nao2 = (size_t)it.p->nao * it.p->nao;
        it.n_k = s.with_k ? (s.hermi == 0 ? 2 * it.n_dm : it.n_dm) : 0;
        it.n_j = (s.with_j && s.hermi != 2) ? it.n_dm : 0;
        it.n_ka = it.n_k ? it.n_dm : 0;
        it.need_t = s.with_k && s.hermi == 0;
        it.n_kp = pair_k && !s.grad ? it.n_k / 2 : 0;
        // a gradient build reads the densities but keeps no J/K accumulators
        if (!s.grad) acc += align256((size_t)it.n_k * nao2 * 8) + align256((size_t)it.n_j * nao2 * 8);
    }
    const size_t jx_bytes = jx ? align256((size_t)items[0].n_j * items[0].p->nx_total * 8) : 0;
    acc += jx_bytes;               // the x-space J, cleared with the accumulators
    need = acc + jx_bytes;         // and the x-space densities
    for (const Item &it : items) {
        const size_t nao2 = (size_t)it.p->nao * it.p->nao;
        need += align256((size_t)it.n_j * nao2 * 8) +
                align256(it.need_t ? (size_t)it.n_dm * nao2 * 8 : 0) +
                align256((size_t)it.n_kp * nao2 * 16) +
                align256((size_t)it.p->nbas * it.p->nbas * 4);
    }
    need += align256((size_t)n * 4);
    char *ws = nullptr;
    if (ws_ext) {
        if (need > ws_ext_size)
            return fail(JK_ERR_SCRATCH, std::string(who) + ": this build needs " + std::to_string(need) +
                                          " bytes of scratch, the library's static scratch holds " +
                                          std::to_string(ws_ext_size) +
                                          " (use jk_build for larger molecules or more densities)");
        ws = ws_ext;
    } else {
        if (need > E.ws_size) {
            if (no_alloc) return fail(JK_ERR_SCRATCH, std::string(who) + ": workspace beyond reservation");
            RC(engine_idle(E));
            cudaFree(E.d_ws);
            E.d_ws = nullptr;
            E.ws_size = 0;
            E.alloc_gen++;
            if (cudaMalloc(&E.d_ws, need) != cudaSuccess) {
                cudaGetLastError();
                return fail(JK_ERR_NOMEM, std::string(who) + ": cannot allocate " +
                                              std::to_string(need) + " bytes of workspace");
            }
            E.ws_size = need;
        }
        ws = E.d_ws;
    }
    size_t o = 0;
    for (Item &it : items) {
        const size_t nao2 = (size_t)it.p->nao * it.p->nao;
        it.Kh = (double *)(ws + o);
        o += s.grad ? 0 : align256((size_t)it.n_k * nao2 * 8);
        it.Jh = (double *)(ws + o);
        o += s.grad ? 0 : align256((size_t)it.n_j * nao2 * 8);
    }
    E.jx = jx;
    E.jx_jonly = !s.with_k;
    E.md_ok = jx && !s.with_k && s.nterm == 1 && s.omega[0] == 0.0 && items[0].n_j <= JK_MD_DENS;
    E.jx_acc = jx ? (double *)(ws + o) : nullptr;
    o += jx_bytes;
    for (Item &it : items) {
        const size_t nao2 = (size_t)it.p->nao * it.p->nao;
        it.dsJ = (double *)(ws + o);
        o += align256((size_t)it.n_j * nao2 * 8);
        it.DT = (double *)(ws + o);
        o += align256(it.need_t ? (size_t)it.n_dm * nao2 * 8 : 0);
        it.dmK2 = it.n_kp ? (double2 *)(ws + o) : nullptr;
        o += align256((size_t)it.n_kp * nao2 * 16);
        it.dmc = (float *)(ws + o);
        o += align256((size_t)it.p->nbas * it.p->nbas * 4);
    }
    E.jx_dens = jx ? (double *)(ws + o) : nullptr;
    o += jx_bytes;
    if (jx) {
        E.jx_plan = items[0].p;
        E.jx_ds = items[0].dsJ;
        E.jx_Jh = items[0].Jh;
        E.jx_nj = items[0].n_j;
    }
    float *dm_max = (float *)(ws + o);
    for (int i = 0; i < n; ++i) items[i].dm_max = dm_max + i;
    E.ws = ws;
    E.acc_bytes = acc;
    E.nitems = n;

    // ---- class views ----
    const float log_mixed = s.mixed_threshold > 0 ? (float)std::log(s.mixed_threshold) : -INFINITY;
    E.mixed = s.mixed_threshold > 0;
    E.grad = s.grad ? s.grad_out : nullptr;
    E.grad_bytes = s.grad ? (size_t)items[0].p->natm * 3 * sizeof(double) : 0;
    E.grad_wj = s.grad_wj;
    E.grad_wk = s.grad_wk;
    E.grad_atom = s.grad ? items[0].p->d_sh_atom : nullptr;
    E.nterm = s.nterm;
    for (int t = 0; t < 2; ++t) {
        const bool on = t < s.nterm;
        E.op_coef[t] = on ? s.coef[t] : 0.0;
        E.op_inv_om2[t] = on && s.omega[t] > 0 ? 1.0 / (s.omega[t] * s.omega[t]) : 0.0;
    }
    bool any = false;
    for (const Item &it : items) any = any || it.n_j || it.n_k;
    std::vector<PlanView> views;
    std::vector<int> row0;
    long long max_rows = 0;
    for (int c = 0; c < JK_NCLASSES; ++c) {
        const ClassEntry &ce = jk_class_table[c];
        const int A = ce.bra_class, B = ce.ket_class;
        E.cls_view0[c] = (int)views.size();
        long long rows = 0;
        int maxprim = 0;
        for (const Item &it : items) {
            if (!any) break;
            const jk_plan *p = it.p;
            const int nbra = p->pc_off[A + 1] - p->pc_off[A];
            const int nket = p->pc_off[B + 1] - p->pc_off[B];
            const int nsub = p->sub_off[B + 1] - p->sub_off[B];
            if (nbra == 0 || nket == 0) continue;
            PlanView v;
            v.bra = p->d_pairs + p->pc_off[A];
            v.ket = p->d_pairs + p->pc_off[B];
            v.sub = p->d_subs + p->sub_off[B];
            v.prim = p->d_prim;
            v.prim_soa = p->d_prim_soa;
            v.prim32 = p->d_prim32;
            v.dm_cond = it.dmc;
            v.dm_max = it.dm_max;
            v.dmK = it.dm;
            v.dmKT = it.DT;
            v.dmK2 = it.dmK2;
            v.dsJ = it.dsJ;
            v.Kh = it.Kh;
            v.Jh = it.Jh;
            v.nbra = nbra;
            v.nket = nket;
            v.nsub = nsub;
            v.same_class = A == B;
            v.nbas = p->nbas;
            v.nao = p->nao;
            v.n_ka = it.n_ka;
            v.n_k = it.n_k;
            v.n_j = it.n_j;
            v.log_tol = p->build_log_tol;
            v.mixed_log_thr = log_mixed;
            v.row0 = (int)rows;
            rows += (long long)nbra * nsub;
            if (rows > INT_MAX) return fail(JK_ERR_ARG, std::string(who) + ": too many task rows");
            maxprim = std::max(maxprim, p->pc_maxprim[A]);
            views.push_back(v);
            row0.push_back(v.row0);
        }
        E.cls_nview[c] = (int)views.size() - E.cls_view0[c];
        E.cls_rows[c] = (int)rows;
        E.cls_maxprim[c] = maxprim;
        max_rows = std::max(max_rows, rows);
    }
    // launches per class: JK_VTAB views each, every launch with its counter
    int ncounters = 0;
    for (int c = 0; c < JK_NCLASSES; ++c) {
        E.cls_nlaunch[c] = (E.cls_nview[c] + JK_VTAB - 1) / JK_VTAB;
        E.cls_cnt0[c] = ncounters;
        ncounters += E.cls_nlaunch[c];
    }
    E.ncounters = ncounters;
    if (ncounters > E.counter_cap) {
        if (no_alloc) return fail(JK_ERR_SCRATCH, std::string(who) + ": counters beyond reservation");
        RC(engine_idle(E));
        cudaFree(E.d_counters);
        E.d_counters = nullptr;
        E.counter_cap = 0;
        E.alloc_gen++;
        if (cudaMalloc(&E.d_counters, ncounters * sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            return fail(JK_ERR_NOMEM, std::string(who) + ": cannot allocate the task counters");
        }
        E.counter_cap = ncounters;
    }
    // ---- density preparation, screening and assembly descriptors ----
    std::vector<TileOp> pre, post;
    std::vector<CondItem> cond;
    std::vector<PairOp> pairs;
    long long pre_tiles = 0, post_tiles = 0, cblk = 0, pblk = 0;
    auto op = [](const double *a, const double *b, double *out, double *outT, double f, int nao,
                 int nd, long long &tiles) {
        TileOp t;
        t.a = a;
        t.b = b;
        t.out = out;
        t.outT = outT;
        t.f = f;
        t.n = nao;
        t.nd = nd;
        t.nt = (nao + 31) / 32;
        t.tile0 = tiles;
        tiles += (long long)nd * t.nt * t.nt;
        return t;
    };
    for (const Item &it : items) {
        const int nao = it.p->nao;
        const size_t nao2 = (size_t)nao * nao;
        if (it.n_j || it.need_t)   // D + D^T for J, D^T for the K of hermi 0
            pre.push_back(op(it.dm, it.dm, it.n_j ? it.dsJ : nullptr, it.need_t ? it.DT : nullptr,
                             1.0, nao, it.n_dm, pre_tiles));
        if (s.with_j && !s.grad)   // J = J_h + J_h^T (zero for hermi 2)
            post.push_back(it.n_j ? op(it.Jh, it.Jh, it.vj, nullptr, 1.0, nao, it.n_dm, post_tiles)
                                  : op(nullptr, nullptr, it.vj, nullptr, 0.0, nao, it.n_dm, post_tiles));
        if (s.with_k && !s.grad) { // K = K_h(D) + K_h(D^T)^T, or K_h +- K_h^T
            if (s.hermi == 0)
                post.push_back(op(it.Kh, it.Kh + (size_t)it.n_dm * nao2, it.vk, nullptr, 1.0, nao,
                                  it.n_dm, post_tiles));
            else
                post.push_back(op(it.Kh, it.Kh, it.vk, nullptr, s.hermi == 2 ? -1.0 : 1.0, nao,
                                  it.n_dm, post_tiles));
        }
        CondItem ci;
        ci.dm = it.dm;
        ci.sh_ao = it.p->d_sh_ao;
        ci.sh_nf = it.p->d_sh_nf;
        ci.dmc = it.dmc;
        ci.dm_max = it.dm_max;
        ci.n_dm = it.n_dm;
        ci.nao = nao;
        ci.nbas = it.p->nbas;
        ci.nt = (it.p->nbas + 15) / 16;
        ci.blk0 = cblk;
        ci.q_drop = it.p->q_drop_max;
        ci.q_max = it.p->q_max;
        ci.log_tol = it.p->build_log_tol;
        ci.pad = 0;
        cblk += (long long)ci.nt * ci.nt;
        cond.push_back(ci);
        // K density d is dm[d] for d < n_ka, then the transposes DT[d - n_ka]
        auto kd = [&](int d) { return d < it.n_ka ? it.dm + d * nao2 : it.DT + (d - it.n_ka) * nao2; };
        for (int q = 0; q < it.n_kp; ++q) {
            PairOp po;
            po.a = kd(2 * q);
            po.b = kd(2 * q + 1);
            po.out = it.dmK2 + q * nao2;
            po.n = (long long)nao2;
            po.blk0 = pblk;
            pblk += ((long long)nao2 + JK_PAIR_THREADS - 1) / JK_PAIR_THREADS;
            pairs.push_back(po);
        }
    }
    if (pre_tiles > INT_MAX || post_tiles > INT_MAX || cblk > INT_MAX || pblk > INT_MAX)
        return fail(JK_ERR_ARG, std::string(who) + ": build too large");
    E.npre = (int)pre.size();
    E.npost = (int)post.size();
    E.npair = (int)pairs.size();
    E.pair_blocks = pblk;
    E.pre_tiles = pre_tiles;
    E.post_tiles = post_tiles;
    E.cond_blocks = cblk;
    E.off_views = 0;
    E.off_row0 = E.off_views + align256(views.size() * sizeof(PlanView));
    E.off_pre = E.off_row0 + align256(row0.size() * sizeof(int));
    E.off_post = E.off_pre + align256(pre.size() * sizeof(TileOp));
    E.off_cond = E.off_post + align256(post.size() * sizeof(TileOp));
    E.off_pair = E.off_cond + align256(cond.size() * sizeof(CondItem));
    const size_t total = E.off_pair + align256(pairs.size() * sizeof(PairOp));
    E.blob.assign(total, 0);
    put(E.blob, E.off_views, views);
    put(E.blob, E.off_row0, row0);
    put(E.blob, E.off_pre, pre);
    put(E.blob, E.off_post, post);
    put(E.blob, E.off_cond, cond);
    put(E.blob, E.off_pair, pairs);
    RC(engine_reserve_rows(E, std::max<long long>(1, max_rows), no_alloc, who));
    RC(engine_reserve_blob(E, total, no_alloc, who));
    return JK_OK;
}

// Orders this build after the engine's previous one when that ran on
// another stream, and uploads the descriptors unless the device already
// holds the same.  Not for a capturing stream.
static int engine_upload(Engine &E, cudaStream_t st)
{
    if (E.done_ev_rec && E.done_stream != st) CK(cudaStreamWaitEvent(st, E.done_ev, 0));
    if (E.blob == E.blob_dev) return JK_OK;
    if (E.blob_ev_rec) CK(cudaEventSynchronize(E.blob_ev));   // staging copy free again
    std::memcpy(E.h_blob, E.blob.data(), E.blob.size());
    CK(cudaMemcpyAsync(E.d_blob, E.h_blob, E.blob.size(), cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(E.blob_ev, st));
    E.blob_ev_rec = true;
    E.blob_dev = E.blob;
    return JK_OK;
}

// the task-row buffers of class stream s
static int *rows_of(const Engine &E, int s) { return E.d_rows + (size_t)s * 4 * E.max_rows; }

// launch l of class c, on class stream s: views [l JK_VTAB, ...) of the class
static ClassArgs class_args(const Engine &E, int c, int l, int s, const PlanView **host_views)
{
    const PlanView *hv = (const PlanView *)(E.blob.data() + E.off_views) + E.cls_view0[c];
    ClassArgs a;
    a.views = (const PlanView *)(E.d_blob + E.off_views) + E.cls_view0[c];
    a.view_row0 = (const int *)(E.d_blob + E.off_row0) + E.cls_view0[c];
    a.nviews = E.cls_nview[c];
    a.nrows = E.cls_rows[c];
    a.view_begin = l * JK_VTAB;
    a.nvl = std::min(JK_VTAB, a.nviews - a.view_begin);
    a.row_begin = hv[a.view_begin].row0;
    a.row_end = a.view_begin + a.nvl < a.nviews ? hv[a.view_begin + a.nvl].row0 : a.nrows;
    a.max_bra_prim = E.cls_maxprim[c];
    a.mixed = E.mixed && E.tune[c].fp32;
    a.mixed_tab = 0;
    a.shard_rank = E.shard_rank;
    a.shard_size = E.shard_size;
    // batched register-form classes take a bra's sub-lists as one task range
    // (the batched kernel walks them); a single plan's keep per-sub-list
    // tasks, whose count fills the GPU for a small molecule
    a.grouped = jk_class_table[c].form == 0 && E.cls_nview[c] > 1;
    // the J engine: every class of a J-only build; with K, the team-form
    // classes (J from the x-space contraction, K from the transfers)
    // (2: a J-only build, whose register-form kernel has no K path)
    a.jx = E.jx && (E.jx_jonly || jk_class_table[c].form == 1 || E.jx_reg)
               ? (E.jx_jonly ? 2 : 1)
               : 0;
    // 3: McMurchie-Davidson J in place of the J engine (the class's choice)
    if (a.jx == 2 && E.md_ok && jk_class_table[c].md && E.tune[c].jmd) a.jx = 3;
    a.jx_dens = E.jx_dens;
    a.jx_acc = E.jx_acc;
    a.grad = E.grad;
    a.sh_atom = E.grad_atom;
    a.natm = E.grad ? (int)(E.grad_bytes / (3 * sizeof(double))) : 0;
    a.grad_wj = E.grad_wj;
    a.grad_wk = E.grad_wk;
    a.nterm = E.nterm;
    for (int t = 0; t < 2; ++t) {
        a.op_coef[t] = E.op_coef[t];
        a.op_inv_om2[t] = E.op_inv_om2[t];
    }
    a.rys = E.rys;
    a.rys32 = E.rys32;
    a.counter = E.d_counters + E.cls_cnt0[c] + l;
    a.chunk = E.d_chunk + c;
    a.row_ncand = rows_of(E, s);
    a.row_prefix = rows_of(E, s) + 2 * E.max_rows;
    a.nquartets = E.d_nq + c;
    a.nprimq = E.d_nq + JK_NCLASSES + c;
    a.nquartets32 = E.d_nq + 2 * JK_NCLASSES + c;
    *host_views = hv + a.view_begin;
    return a;
}

// Sets the launch attributes of every class kernel the prepared build uses
// (nothing is launched): a stream capture then changes no kernel state.
static int engine_configure(Engine &E)
{
    char msg[256] = {0};
    LaunchCfg cfg;
    cfg.stream = nullptr;
    cfg.device = E.device;
    cfg.num_sms = E.num_sms;
    cfg.blocks_per_sm = 0;
    cfg.configure_only = 1;
    cfg.msg = msg;
    std::lock_guard<std::mutex> lock(g_launch_mutex);
    for (int c = 0; c < JK_NCLASSES; ++c) {
        for (int l = 0; l < E.cls_nlaunch[c]; ++l) {
            const PlanView *hv = nullptr;
            const ClassArgs a = class_args(E, c, l, 0, &hv);
            const int rc = jk_class_table[c].launch(a, hv, cfg);
            if (rc) return fail(JK_ERR_CUDA, std::string("class kernel configuration failed: ") + msg);
        }
    }
    return JK_OK;
}

// J engine: the pair transforms of every pair class of the build's plan,
// densities (post = false) or J (post = true)
static int jx_pairs(Engine &E, cudaStream_t st, bool post)
{
    const jk_plan *p = E.jx_plan;
    for (int t = 0; t < JK_NPAIR_TABLE; ++t) {
        const PairEntry &pe = jk_pair_table[t];
        PairArgs a;
        a.pairs = p->d_pairs + p->pc_off[pe.pair_class];
        a.npairs = p->pc_off[pe.pair_class + 1] - p->pc_off[pe.pair_class];
        if (a.npairs == 0) continue;
        a.n_j = E.jx_nj;
        a.nao = p->nao;
        a.ds = E.jx_ds;
        a.Jh = E.jx_Jh;
        a.dt = E.jx_dens;
        a.jx = E.jx_acc;
        const int rc = post ? pe.post(a, st) : pe.dens(a, st);
        if (rc) return fail(JK_ERR_CUDA, std::string("J engine pair kernel: ") +
                                             cudaGetErrorString((cudaError_t)rc));
        E.launches++;
    }
    return JK_OK;
}

// The launch stream of a prepared build (stream operations only, so that it
// can be captured).
static int engine_launch(Engine &E, cudaStream_t st, bool timing)
{
    E.launches = 0;
    if (timing) std::fill(E.ev_used.begin(), E.ev_used.end(), 0);
    const TileOp *d_pre = (const TileOp *)(E.d_blob + E.off_pre);
    const TileOp *d_post = (const TileOp *)(E.d_blob + E.off_post);
    const CondItem *d_cond = (const CondItem *)(E.d_blob + E.off_cond);
    if (E.acc_bytes) CK(cudaMemsetAsync(E.ws, 0, E.acc_bytes, st));
    if (E.grad) CK(cudaMemsetAsync(E.grad, 0, E.grad_bytes, st));
    if (E.npre) {
        tile_op_kernel<<<(unsigned)E.pre_tiles, dim3(32, 8), 0, st>>>(d_pre, E.npre);
        CK(cudaGetLastError());
        E.launches++;
    }
    dm_cond_kernel<<<(unsigned)E.cond_blocks, dim3(16, 16), 0, st>>>(d_cond, E.nitems);
    CK(cudaGetLastError());
    dm_max_kernel<<<E.nitems, 256, 0, st>>>(d_cond, E.d_error);
    CK(cudaGetLastError());
    E.launches += 2;
    if (E.npair) {   // after the transposes of the pre step
        pair_dens_kernel<<<(unsigned)E.pair_blocks, JK_PAIR_THREADS, 0, st>>>(
            (const PairOp *)(E.d_blob + E.off_pair), E.npair);
        CK(cudaGetLastError());
        E.launches++;
    }
    if (E.jx) RC(jx_pairs(E, st, false));   // x-space densities of every pair
    if (E.ncounters) CK(cudaMemsetAsync(E.d_counters, 0, E.ncounters * sizeof(int), st));
    CK(cudaMemsetAsync(E.d_nq, 0, 3 * JK_NCLASSES * sizeof(unsigned long long), st));
    char msg[256] = {0};
    LaunchCfg cfg;
    cfg.device = E.device;
    cfg.num_sms = E.num_sms;
    cfg.configure_only = 0;
    cfg.msg = msg;
    // fork the class streams off the build's stream (also inside a capture);
    // with serialised per-class timing (mode 1) one stream, so that each
    // class's events bracket its own kernels only; mode 2 keeps the class
    // streams and records each class's events on its own stream
    const int ns = timing && E.timing_mode == 1 ? 1 : JK_CLASS_STREAMS;
    cudaStream_t cs[JK_CLASS_STREAMS];
    cs[0] = st;
    if (ns > 1) CK(cudaEventRecord(E.ev_fork, st));
    for (int s = 1; s < ns; ++s) {
        cs[s] = E.side[s - 1];
        CK(cudaStreamWaitEvent(cs[s], E.ev_fork, 0));
    }
    int nactive = 0;
    for (int c = 0; c < JK_NCLASSES; ++c) {
        const int rows = E.cls_rows[c];
        if (!E.cls_nview[c] || rows == 0) continue;
        const int si = nactive++ % ns;
        const cudaStream_t cst = cs[si];
        int *rb = rows_of(E, si);
        int *chunks = rb + E.max_rows;
        int *prefix = rb + 2 * E.max_rows;
        int *cand_prefix = rb + 3 * E.max_rows;
        void *cub = (char *)E.d_cub + si * E.cub_stride;
        const ClassEntry &ce = jk_class_table[c];
        const PlanView *hv = nullptr;
        const ClassArgs a = class_args(E, c, 0, si, &hv);
        if (timing) CK(cudaEventRecord(E.ev[2 * c], cst));
        // task list: candidates per row, a task size giving about
        // tasks_per_sm tasks per SM, chunks per row, prefix sum of chunks
        task_rows_kernel<<<(rows + 255) / 256, 256, 0, cst>>>(a, rb);
        CK(cudaGetLastError());
        size_t tmp = E.cub_bytes;
        CK(cub::DeviceScan::InclusiveSum(cub, tmp, rb, cand_prefix, rows, cst));
        const int lo = ce.form == 0 ? 128 : 32, hi = ce.form == 0 ? 4096 : 1024;
        const int target = std::max(1, E.tune[c].tasks_per_sm) * E.num_sms;
        task_chunks_kernel<<<(rows + 255) / 256, 256, 0, cst>>>(a, rb, cand_prefix, rows, target,
                                                                lo, hi, E.d_chunk + c, chunks);
        CK(cudaGetLastError());
        tmp = E.cub_bytes;
        CK(cub::DeviceScan::InclusiveSum(cub, tmp, chunks, prefix, rows, cst));
        E.launches += 4;
        cfg.stream = cst;
        cfg.blocks_per_sm = E.tune[c].blocks_per_sm;
        for (int l = 0; l < E.cls_nlaunch[c]; ++l) {
            const ClassArgs al = class_args(E, c, l, si, &hv);
            int rc;
            {
                std::lock_guard<std::mutex> lock(g_launch_mutex);
                rc = ce.launch(al, hv, cfg);
            }
            if (rc != 0)
                return fail(JK_ERR_CUDA, std::string("class kernel launch failed: ") + msg + " " +
                                             cudaGetErrorString((cudaError_t)rc));
            E.launches++;
        }
        if (timing) {
            CK(cudaEventRecord(E.ev[2 * c + 1], cst));
            E.ev_used[c] = 1;
        }
    }
    // join the class streams back into the build's stream
    for (int s = 1; s < ns; ++s) {
        CK(cudaEventRecord(E.ev_join[s - 1], cs[s]));
        CK(cudaStreamWaitEvent(st, E.ev_join[s - 1], 0));
    }
    if (E.jx) RC(jx_pairs(E, st, true));    // x-space J into the half-J accumulators
    if (E.npost) {
        tile_op_kernel<<<(unsigned)E.post_tiles, dim3(32, 8), 0, st>>>(d_post, E.npost);
        CK(cudaGetLastError());
        E.launches++;
    }
    return JK_OK;
}

static int engine_finish(Engine &E, cudaStream_t st)
{
    CK(cudaEventRecord(E.done_ev, st));
    E.done_ev_rec = true;
    E.done_stream = st;
    E.last_stream = st;
    return JK_OK;
}

// prepare, upload and launch a build outside any capture
static int engine_build(Engine &E, std::vector<Item> &items, const Spec &s, cudaStream_t st,
                        char *ws_ext, size_t ws_ext_size, bool no_alloc, const char *who)
{
    RC(engine_prepare(E, items, s, ws_ext, ws_ext_size, no_alloc, who));
    RC(engine_upload(E, st));
    RC(engine_launch(E, st, E.timing));
    return engine_finish(E, st);
}

static int engine_sync(Engine &E, cudaStream_t st, const char *who)
{
    CK(cudaStreamSynchronize(st));
    int err[2] = {0, 0};
    CK(cudaMemcpy(err, E.d_error, sizeof(err), cudaMemcpyDeviceToHost));
    if (err[0]) {
        CK(cudaMemset(E.d_error, 0, sizeof(err)));
        if (err[0] == JK_ERR_RANGE)
            return fail(JK_ERR_RANGE, std::string(who) + ": density elements of item " +
                                          std::to_string(err[1]) +
                                          " exceed the range the plan was built for "
                                          "(shell pairs it dropped would pass the screening)");
        return fail(JK_ERR_DEVICE, std::string(who) + ": kernel error flag " + std::to_string(err[0]));
    }
    return JK_OK;
}

static int engine_counts(Engine &E, unsigned long long *quartets, unsigned long long *prim_quartets,
                         unsigned long long *quartets_f32, int ncounts, int *nclasses)
{
    if (nclasses) *nclasses = JK_NCLASSES;
    if (!quartets && !prim_quartets && !quartets_f32) return JK_OK;
    CK(cudaStreamSynchronize(E.last_stream));
    std::vector<unsigned long long> h(3 * JK_NCLASSES);
    CK(cudaMemcpy(h.data(), E.d_nq, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    for (int k = 0; k < ncounts && k < JK_NCLASSES; ++k) {
        if (quartets) quartets[k] = h[k];
        if (prim_quartets) prim_quartets[k] = h[JK_NCLASSES + k];
        if (quartets_f32) quartets_f32[k] = h[2 * JK_NCLASSES + k];
    }
    return JK_OK;
}

static int engine_set_timing(Engine &E, int enable)
{
    if (enable && E.ev.empty()) {
        E.ev.resize(2 * JK_NCLASSES);
        for (auto &e : E.ev) CK(cudaEventCreate(&e));
        E.ev_used.assign(JK_NCLASSES, 0);
    }
    if (enable < 0 || enable > 2) return fail(JK_ERR_ARG, "timing mode must be 0, 1 or 2");
    E.timing = enable != 0;
    E.timing_mode = enable;
    return JK_OK;
}

static int engine_class_ms(Engine &E, float *ms, int ncounts, int *launches)
{
    if (launches) *launches = E.launches;
    if (!ms) return JK_OK;
    CK(cudaStreamSynchronize(E.last_stream));
    for (int c = 0; c < ncounts && c < JK_NCLASSES; ++c) {
        ms[c] = 0.f;
        if (E.timing && c < (int)E.ev_used.size() && E.ev_used[c])
            CK(cudaEventElapsedTime(&ms[c], E.ev[2 * c], E.ev[2 * c + 1]));
    }
    return JK_OK;
}

static int engine_set_tuning(Engine &E, int cls, int tasks_per_sm, int blocks_per_sm, int fp32)
{
    if (cls < -1 || cls >= JK_NCLASSES) return fail(JK_ERR_ARG, "tuning: no such class");
    if (tasks_per_sm < 0 || blocks_per_sm < 0) return fail(JK_ERR_ARG, "tuning: negative value");
    if (cls == -1) {
        engine_defaults(E);
    } else {
        const int def = jk_class_table[cls].form == 0 ? 64 : 16;
        E.tune[cls].tasks_per_sm = tasks_per_sm ? tasks_per_sm : def;
        E.tune[cls].blocks_per_sm = blocks_per_sm;
        E.tune[cls].fp32 = fp32 < 0 ? jk_class_table[cls].fp32_default : fp32 != 0;
    }
    E.tune_gen++;
    return JK_OK;
}

// ---------------------------------------------------------------------------
// plans
// ---------------------------------------------------------------------------
static void free_plan(jk_plan *p)
{
    cudaFree(p->d_shells);
    cudaFree(p->d_basis);
    cudaFree(p->d_prim);
    cudaFree(p->d_prim_soa);
    cudaFree(p->d_prim32);
    cudaFree(p->d_pairs);
    cudaFree(p->d_sh_ao);
    cudaFree(p->d_sh_nf);
    cudaFree(p->d_io);
    cudaFree(p->d_subs);
    engine_free(p->eng);
}

template <class T>
static cudaError_t upload(T **dst, const std::vector<T> &src, cudaStream_t st, size_t *bytes_out)
{
    const size_t bytes = std::max<size_t>(1, src.size()) * sizeof(T);
    cudaError_t e = cudaMalloc((void **)dst, bytes);
    if (e != cudaSuccess) return e;
    if (bytes_out) *bytes_out += bytes;
    if (!src.empty())
        e = cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, st);
    return e;
}

// owns the private stream and the temporaries of a plan construction
struct PlanScratch {
    cudaStream_t st = nullptr;
    int4 *d_rec = nullptr, *d_cand = nullptr;
    float *d_q = nullptr;
    ~PlanScratch()
    {
        if (st) {
            cudaStreamSynchronize(st);
            cudaFreeAsync(d_rec, st);
            cudaFreeAsync(d_cand, st);
            cudaFreeAsync(d_q, st);
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    }
};

static int plan_create(const int *atm, int natm, const int *bas, int nbas_user, const double *env,
                       const int *ao_loc, double tol, int device, jk_plan *p)
{
    if (!atm || !bas || !env || !ao_loc || natm <= 0 || nbas_user <= 0)
        return fail(JK_ERR_ARG, "jk_plan_create: null array or empty molecule");
    if (!(tol > 0.0)) return fail(JK_ERR_ARG, "jk_plan_create: direct_scf_tol must be > 0");
    p->device = device;
    p->tol = tol;
    p->log_tol = (float)std::log(tol);
    p->build_tol = tol;
    p->build_log_tol = p->log_tol;
    p->nbas_user = nbas_user;
    p->natm = natm;
    RC(engine_init(p->eng, device));

    // ---- shells (general contractions expanded, contraction-major) ----
    std::vector<ShellDev> shells;
    std::vector<double> basis;
    for (int s = 0; s < nbas_user; ++s) {
        const int *b = bas + s * 8;
        const int ia = b[0], l = b[1], nprim = b[2], nctr = b[3];
        if (ia < 0 || ia >= natm) return fail(JK_ERR_ARG, "bas: atom index out of range");
        if (l < 0 || l > 3)
            return fail(JK_ERR_UNSUPPORTED, "shell " + std::to_string(s) + ": l = " +
                                                std::to_string(l) + " (the engine handles l <= 3)");
        if (nprim < 1 || nctr < 1) return fail(JK_ERR_ARG, "bas: empty shell");
        if (ao_loc[s + 1] - ao_loc[s] != nctr * ncart(l))
            return fail(JK_ERR_ARG, "ao_loc is not the Cartesian AO layout of bas (shell " +
                                        std::to_string(s) + ")");
        const double *xyz = env + atm[ia * 6 + 1];
        for (int c = 0; c < nctr; ++c) {
            ShellDev sd;
            sd.x = xyz[0]; sd.y = xyz[1]; sd.z = xyz[2];
            sd.l = l;
            sd.nprim = nprim;
            sd.exp_off = (int)basis.size();
            for (int k = 0; k < nprim; ++k) basis.push_back(env[b[5] + k]);
            sd.coef_off = (int)basis.size();
            for (int k = 0; k < nprim; ++k) basis.push_back(env[b[6] + c * nprim + k] * common_fac(l));
            shells.push_back(sd);
            p->sh_l.push_back(l);
            p->sh_ao.push_back(ao_loc[s] + c * ncart(l));
            p->sh_user.push_back(s);
            p->sh_atom.push_back(ia);
        }
        if (nctr > 1) p->expanded = true;
    }
    const int nbas = (int)shells.size();
    p->nbas = nbas;
    p->nao = ao_loc[nbas_user];

    // ---- candidate shell pairs and their kept primitive pairs ----
    std::vector<int4> cand;          // ish, jsh, prim0, nprim
    std::vector<int4> rec;           // ish, jsh, pi, pj
    for (int i = 0; i < nbas; ++i) {
        for (int j = 0; j < nbas; ++j) {
            const int li = shells[i].l, lj = shells[j].l;
            if (!(li > lj || (li == lj && i >= j))) continue;
            const double dx = shells[i].x - shells[j].x, dy = shells[i].y - shells[j].y,
                         dz = shells[i].z - shells[j].z;
            const double rr = dx * dx + dy * dy + dz * dz;
            const int r0 = (int)rec.size();
            for (int pi = 0; pi < shells[i].nprim; ++pi) {
                const double ai = basis[shells[i].exp_off + pi];
                for (int pj = 0; pj < shells[j].nprim; ++pj) {
                    const double aj = basis[shells[j].exp_off + pj];
                    if (ai * aj / (ai + aj) * rr > JK_PRIM_EXP_CUTOFF) continue;
                    rec.push_back(make_int4(i, j, pi, pj));
                }
            }
            const int n = (int)rec.size() - r0;
            if (n > 0) cand.push_back(make_int4(i, j, r0, n));
        }
    }
    if ((long long)rec.size() > (1ll << 31) - 1) return fail(JK_ERR_ARG, "molecule too large");

    // the construction runs on a private stream, so that it does not wait
    // for (or hold up) builds of other plans on the caller's streams
    PlanScratch tmp;
    CK(cudaStreamCreateWithFlags(&tmp.st, cudaStreamNonBlocking));
    const cudaStream_t st = tmp.st;
    CK(upload(&p->d_shells, shells, st, &p->table_bytes));
    CK(upload(&p->d_basis, basis, st, &p->table_bytes));
    CK(cudaMallocAsync(&tmp.d_rec, std::max<size_t>(1, rec.size()) * sizeof(int4), st));
    CK(cudaMallocAsync(&tmp.d_cand, std::max<size_t>(1, cand.size()) * sizeof(int4), st));
    CK(cudaMallocAsync(&tmp.d_q, std::max<size_t>(1, cand.size()) * sizeof(float), st));
    if (!rec.empty())
        CK(cudaMemcpyAsync(tmp.d_rec, rec.data(), rec.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
    if (!cand.empty())
        CK(cudaMemcpyAsync(tmp.d_cand, cand.data(), cand.size() * sizeof(int4), cudaMemcpyHostToDevice,
                           st));
    const size_t prim_bytes = std::max<size_t>(1, rec.size()) * JK_PRIM_STRIDE * sizeof(double);
    CK(cudaMalloc(&p->d_prim, prim_bytes));
    const size_t prim32_bytes = std::max<size_t>(1, rec.size()) * JK_PRIM32_STRIDE * sizeof(float);
    CK(cudaMalloc(&p->d_prim32, prim32_bytes));
    p->table_bytes += prim_bytes + prim32_bytes;

    if (!rec.empty()) {
        const int nt = 256;
        prim_pair_fill_kernel<<<(unsigned)((rec.size() + nt - 1) / nt), nt, 0, st>>>(
            tmp.d_rec, (long long)rec.size(), p->d_shells, p->d_basis, p->d_prim);
        CK(cudaGetLastError());
        prim32_fill_kernel<<<(unsigned)((rec.size() + nt - 1) / nt), nt, 0, st>>>(
            p->d_prim, (long long)rec.size(), p->d_prim32);
        CK(cudaGetLastError());
        schwarz_kernel<<<(unsigned)((cand.size() + 127) / 128), 128, 0, st>>>(
            tmp.d_cand, (int)cand.size(), p->d_shells, p->d_prim, p->eng.rys, tmp.d_q);
        CK(cudaGetLastError());
    }
    std::vector<float> q(cand.size());
    if (!cand.empty())
        CK(cudaMemcpyAsync(q.data(), tmp.d_q, q.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));

    // ---- keep, classify, sort ----
    float qmax = -INFINITY;
    for (float v : q) qmax = std::max(qmax, v);
    p->q_max = qmax;
    p->q_full.assign((size_t)nbas * nbas, -INFINITY);
    std::vector<std::vector<int>> byclass(NPAIR_CLASSES);
    for (size_t c = 0; c < cand.size(); ++c) {
        const int i = cand[c].x, j = cand[c].y;
        p->q_full[(size_t)i * nbas + j] = q[c];
        p->q_full[(size_t)j * nbas + i] = q[c];
        if (!(q[c] > -INFINITY)) continue;
        if (q[c] + qmax + PLAN_DM_MARGIN <= p->log_tol) {
            p->q_drop_max = std::max(p->q_drop_max, q[c]);
            continue;
        }
        byclass[pair_class(shells[i].l, shells[j].l)].push_back((int)c);
    }
    std::vector<PairRec> recs;
    size_t soa_total = 0, soa_block = 0;   // doubles of the field-major copy
    for (int k = 0; k < NPAIR_CLASSES; ++k) {
        auto &v = byclass[k];
        // primitive-pair count first (sub-lists of equal loop bounds), then
        // the Schwarz bin (descending), then the shells (runs of kets that
        // share their first shell, see JK_QBIN_W)
        std::stable_sort(v.begin(), v.end(), [&](int a, int b) {
            if (cand[a].w != cand[b].w) return cand[a].w > cand[b].w;
            const float ba = jk_qbin(q[a]), bb = jk_qbin(q[b]);
            if (ba != bb) return ba > bb;
            if (cand[a].x != cand[b].x) return cand[a].x < cand[b].x;
            return cand[a].y < cand[b].y;
        });
        p->pc_off[k] = (int)recs.size();
        p->sub_off[k] = (int)p->subs.size();
        for (size_t t = 0; t < v.size(); ++t) {
            if (t == 0 || cand[v[t]].w != cand[v[t - 1]].w)
                p->subs.push_back(make_int2((int)t, (int)t));
            p->subs.back().y = (int)t + 1;
        }
        int mp = 0;
        size_t sub_start = 0, sub_n = 0;   // the current sub-list's block
        for (size_t t = 0; t < v.size(); ++t) {
            const int c = v[t];
            const int i = cand[c].x, j = cand[c].y;
            if (t == 0 || cand[c].w != cand[v[t - 1]].w) {
                // a new sub-list: its block follows the previous one
                soa_total += sub_n * (size_t)(t ? cand[v[t - 1]].w : 0) * JK_SOA_FIELDS;
                sub_start = t;
                sub_n = 0;
                while (sub_start + sub_n < v.size() && cand[v[sub_start + sub_n]].w == cand[c].w) ++sub_n;
                soa_block = soa_total;
            }
            PairRec r;
            r.ish = i;
            r.jsh = j;
            r.i0 = p->sh_ao[i];
            r.j0 = p->sh_ao[j];
            r.prim0 = cand[c].z;
            r.nprim = cand[c].w;
            r.q = q[c];
            r.xoff = 0;       // set below, once the classes are laid out
            r.soa = (int)std::min<size_t>(soa_block + (t - sub_start), INT_MAX);
            r.soa_n = (int)sub_n;
            r.ABx = shells[i].x - shells[j].x;
            r.ABy = shells[i].y - shells[j].y;
            r.ABz = shells[i].z - shells[j].z;
            mp = std::max(mp, r.nprim);
            recs.push_back(r);
        }
        if (!v.empty()) soa_total += sub_n * (size_t)cand[v.back()].w * JK_SOA_FIELDS;
        p->pc_maxprim[k] = mp;
    }
    if (soa_total > (size_t)INT_MAX) return fail(JK_ERR_ARG, "molecule too large (primitive pairs)");
    p->pc_off[NPAIR_CLASSES] = (int)recs.size();
    // x-space blocks of the J engine in pair order: NX = sum of ncart over
    // the transfer's source levels la..la+lb
    long long xo = 0;
    for (int la = 0; la < 4; ++la)
        for (int lb = 0; lb <= la; ++lb) {
            const int k = pair_class(la, lb);
            int nx = 0;
            for (int L = la; L <= la + lb; ++L) nx += ncart(L);
            for (int r = p->pc_off[k]; r < p->pc_off[k + 1]; ++r) {
                recs[r].xoff = (int)xo;
                xo += nx;
            }
        }
    if (xo > INT_MAX / 8) {   // beyond the J engine's block indices: J from (ij|kl)
        for (PairRec &r : recs) r.xoff = 0;
        xo = 0;
        p->jengine = false;
    }
    p->nx_total = xo;
    for (int k = 0; k < NPAIR_CLASSES; ++k)   // kernels queue ket indices in 28 bits
        if (p->pc_off[k + 1] - p->pc_off[k] >= (1 << 28))
            return fail(JK_ERR_ARG, "molecule too large (shell pairs of one class)");
    p->sub_off[NPAIR_CLASSES] = (int)p->subs.size();
    CK(upload(&p->d_subs, p->subs, st, &p->table_bytes));
    // task rows of one class: the largest (bra class pairs) x (ket class sub-lists)
    long long max_rows = 1;
    for (int A = 0; A < NPAIR_CLASSES; ++A)
        for (int B = 0; B <= A; ++B)
            max_rows = std::max<long long>(
                max_rows, (long long)(p->pc_off[A + 1] - p->pc_off[A]) *
                              (p->sub_off[B + 1] - p->sub_off[B]));
    if (max_rows > (1ll << 31) - 1) return fail(JK_ERR_ARG, "molecule too large (task rows)");
    p->max_rows = max_rows;
    p->npairs = (long long)recs.size();
    CK(upload(&p->d_pairs, recs, st, &p->table_bytes));
    {   // the field-major copy of the primitive records, in ket order
        const size_t bytes = std::max<size_t>(1, soa_total) * sizeof(double);
        CK(cudaMalloc(&p->d_prim_soa, bytes));
        p->table_bytes += bytes;
        if (!recs.empty()) {
            prim_soa_fill_kernel<<<(unsigned)((recs.size() + 127) / 128), 128, 0, st>>>(
                p->d_pairs, (long long)recs.size(), p->d_prim, p->d_prim_soa);
            CK(cudaGetLastError());
        }
    }
    std::vector<int> nf(nbas);
    for (int s = 0; s < nbas; ++s) nf[s] = ncart(shells[s].l);
    CK(upload(&p->d_sh_ao, p->sh_ao, st, &p->table_bytes));
    CK(upload(&p->d_sh_nf, nf, st, &p->table_bytes));
    CK(upload(&p->d_sh_atom, p->sh_atom, st, &p->table_bytes));
    // the plan's own builds (one item) never grow these: jk_build_noalloc
    // relies on it
    RC(engine_reserve_rows(p->eng, max_rows, false, "jk_plan_create"));
    RC(engine_reserve_blob(p->eng, blob_bytes(JK_NCLASSES, 1, 2, 1), false, "jk_plan_create"));
    CK(cudaStreamSynchronize(st));
    return JK_OK;
}

extern "C" int jk_plan_create(const int *atm, int natm, const int *bas, int nbas, const double *env,
                              const int *ao_loc, double direct_scf_tol, int device, jk_plan **out)
{
    if (!out) return fail(JK_ERR_ARG, "jk_plan_create: out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev ||
        device >= JK_MAX_DEVICES)
        return fail(JK_ERR_CUDA, "jk_plan_create: no CUDA device " + std::to_string(device));
    DeviceGuard g(device);
    jk_plan *p = new jk_plan();
    int rc = plan_create(atm, natm, bas, nbas, env, ao_loc, direct_scf_tol, device, p);
    if (rc != JK_OK) {
        free_plan(p);
        delete p;
        return rc;
    }
    *out = p;
    return JK_OK;
}

extern "C" int jk_plan_destroy(jk_plan *plan)
{
    if (!plan) return JK_OK;
    DeviceGuard g(plan->device);
    engine_idle(plan->eng);
    free_plan(plan);
    delete plan;
    return JK_OK;
}

extern "C" int jk_plan_info(const jk_plan *plan, int *nao, long long *npairs)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_plan_info: plan is NULL");
    if (nao) *nao = plan->nao;
    if (npairs) *npairs = plan->npairs;
    return JK_OK;
}

extern "C" int jk_plan_memory(const jk_plan *plan, long long *table_bytes, long long *workspace_bytes)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_plan_memory: plan is NULL");
    if (table_bytes)
        *table_bytes = (long long)(plan->table_bytes +
                                   JK_CLASS_STREAMS * (4 * (size_t)plan->eng.max_rows * sizeof(int) +
                                                       plan->eng.cub_stride) +
                                   plan->eng.blob_cap);
    if (workspace_bytes) *workspace_bytes = (long long)(plan->eng.ws_size + plan->io_size);
    return JK_OK;
}

extern "C" int jk_plan_q_cond(const jk_plan *plan, float *q_host, int nbas)
{
    if (!plan || !q_host) return fail(JK_ERR_ARG, "jk_plan_q_cond: null argument");
    if (plan->expanded || nbas != plan->nbas)
        return fail(JK_ERR_ARG, "jk_plan_q_cond: nbas does not match the plan's shells");
    std::memcpy(q_host, plan->q_full.data(), plan->q_full.size() * sizeof(float));
    return JK_OK;
}

extern "C" int jk_plan_set_shard(jk_plan *plan, int rank, int size)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_plan_set_shard: plan is NULL");
    if (size < 1 || rank < 0 || rank >= size)
        return fail(JK_ERR_ARG, "jk_plan_set_shard: need 0 <= rank < size");
    plan->eng.shard_rank = rank;
    plan->eng.shard_size = size;
    return JK_OK;
}

extern "C" int jk_plan_set_jengine(jk_plan *plan, int on)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_plan_set_jengine: plan is NULL");
    if (on && plan->nx_total == 0 && plan->npairs > 0)
        return fail(JK_ERR_ARG, "jk_plan_set_jengine: the plan's x-space blocks exceed the J "
                                "engine's index range");
    plan->jengine = on != 0;
    return JK_OK;
}

extern "C" int jk_plan_set_tol(jk_plan *plan, double tol)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_plan_set_tol: plan is NULL");
    if (!(tol > 0) || !std::isfinite(tol))
        return fail(JK_ERR_ARG, "jk_plan_set_tol: tol must be positive and finite");
    if (tol < plan->tol) {
        char msg[200];
        snprintf(msg, sizeof(msg),
                 "jk_plan_set_tol: tol %g is below the plan's threshold %g (its pair lists "
                 "would miss quartets): create a new plan", tol, plan->tol);
        return fail(JK_ERR_ARG, msg);
    }
    plan->build_tol = tol;
    plan->build_log_tol = tol == plan->tol ? plan->log_tol : (float)std::log(tol);
    return JK_OK;
}

extern "C" int jk_plan_set_tuning(jk_plan *plan, int cls, int tasks_per_sm, int blocks_per_sm,
                                  int fp32)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_plan_set_tuning: plan is NULL");
    return engine_set_tuning(plan->eng, cls, tasks_per_sm, blocks_per_sm, fp32);
}

extern "C" int jk_plan_set_jmd(jk_plan *plan, int cls, int mode)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_plan_set_jmd: plan is NULL");
    if (cls < -1 || cls >= JK_NCLASSES) return fail(JK_ERR_ARG, "jk_plan_set_jmd: no such class");
    if (mode < -1 || mode > 1) return fail(JK_ERR_ARG, "jk_plan_set_jmd: mode is -1, 0 or 1");
    for (int c = cls < 0 ? 0 : cls; c < (cls < 0 ? JK_NCLASSES : cls + 1); ++c) {
        if (mode == 1 && !jk_class_table[c].md) {
            if (cls >= 0) return fail(JK_ERR_ARG, "jk_plan_set_jmd: the class has no MD J kernel");
            continue;
        }
        plan->eng.tune[c].jmd = mode < 0 ? jk_class_table[c].md_default : mode;
    }
    plan->eng.tune_gen++;
    return JK_OK;
}

// ---------------------------------------------------------------------------
// single-plan builds
// ---------------------------------------------------------------------------
static int build_one(jk_plan *p, const double *dm, int n_dm, int hermi, int with_j, int with_k,
                     double *vj, double *vk, double mixed_threshold, cudaStream_t st, char *ws_ext,
                     size_t ws_ext_size, bool no_alloc, const char *who, const Spec *op = nullptr)
{
    std::vector<Item> items(1);
    items[0].p = p;
    items[0].dm = dm;
    items[0].n_dm = n_dm;
    items[0].vj = vj;
    items[0].vk = vk;
    Spec s = coulomb_spec(hermi, with_j, with_k, mixed_threshold);
    if (op) {
        s.nterm = op->nterm;
        for (int t = 0; t < 2; ++t) {
            s.coef[t] = op->coef[t];
            s.omega[t] = op->omega[t];
        }
    }
    return engine_build(p->eng, items, s, st, ws_ext, ws_ext_size, no_alloc, who);
}

extern "C" int jk_build(jk_plan *plan, const double *dm, int n_dm, int hermi, int with_j,
                        int with_k, double *vj, double *vk, double mixed_threshold, void *stream)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_build: plan is NULL");
    DeviceGuard g(plan->device);
    return build_one(plan, dm, n_dm, hermi, with_j, with_k, vj, vk, mixed_threshold,
                     (cudaStream_t)stream, nullptr, 0, false, "jk_build");
}

extern "C" int jk_build_rs(jk_plan *plan, const double *dm, int n_dm, int hermi, int with_j,
                           int with_k, double *vj, double *vk, double mixed_threshold,
                           double omega, void *stream)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_build_rs: plan is NULL");
    DeviceGuard g(plan->device);
    Spec op = coulomb_spec(hermi, with_j, with_k, mixed_threshold);
    op.omega[0] = omega;
    return build_one(plan, dm, n_dm, hermi, with_j, with_k, vj, vk, mixed_threshold,
                     (cudaStream_t)stream, nullptr, 0, false, "jk_build_rs", &op);
}

extern "C" int jk_build_op(jk_plan *plan, const double *dm, int n_dm, int hermi, int with_j,
                           int with_k, double *vj, double *vk, double mixed_threshold,
                           int n_terms, const double *coef, const double *omega, void *stream)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_build_op: plan is NULL");
    if (n_terms < 1 || n_terms > 2 || !coef || !omega)
        return fail(JK_ERR_ARG, "jk_build_op: n_terms must be 1 or 2, with coef and omega");
    DeviceGuard g(plan->device);
    Spec op = coulomb_spec(hermi, with_j, with_k, mixed_threshold);
    op.nterm = n_terms;
    for (int t = 0; t < n_terms; ++t) {
        op.coef[t] = coef[t];
        op.omega[t] = omega[t];
    }
    return build_one(plan, dm, n_dm, hermi, with_j, with_k, vj, vk, mixed_threshold,
                     (cudaStream_t)stream, nullptr, 0, false, "jk_build_op", &op);
}

extern "C" int jk_grad(jk_plan *plan, const double *dm, int n_dm, double j_factor,
                       double k_factor, double omega, double *grad, void *stream)
{
    if (!plan || !dm || !grad) return fail(JK_ERR_ARG, "jk_grad: null argument");
    if (n_dm < 1 || n_dm > 2) return fail(JK_ERR_ARG, "jk_grad: n_dm must be 1 or 2");
    if (!(omega >= 0) || !std::isfinite(omega))
        return fail(JK_ERR_ARG, "jk_grad: omega must be finite and >= 0");
    if (!std::isfinite(j_factor) || !std::isfinite(k_factor))
        return fail(JK_ERR_ARG, "jk_grad: factors must be finite");
    DeviceGuard g(plan->device);
    std::vector<Item> items(1);
    items[0].p = plan;
    items[0].dm = dm;
    items[0].n_dm = n_dm;
    items[0].vj = items[0].vk = nullptr;
    Spec s = coulomb_spec(1, 1, 1, 0.0);
    s.omega[0] = omega;
    s.grad = 1;
    // W = fac [4 j Dt_ab Dt_cd - 4 k c sum_s (...)], c = 1/4 (one density) or 1/2
    s.grad_wj = 4.0 * j_factor;
    s.grad_wk = 4.0 * k_factor * (n_dm == 1 ? 0.25 : 0.5);
    s.grad_out = grad;
    return engine_build(plan->eng, items, s, (cudaStream_t)stream, nullptr, 0, false, "jk_grad");
}

extern "C" int jk_sync(jk_plan *plan, void *stream)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_sync: plan is NULL");
    DeviceGuard g(plan->device);
    return engine_sync(plan->eng, (cudaStream_t)stream, "jk_sync");
}

// ---------------------------------------------------------------------------
// Allocation-free build.  Its scratch (the half-J/K accumulators, the
// symmetrised and transposed densities and the density screening table)
// lives in this fixed array, which every GPU that loads the library holds
// until the process exits.  Host code must not pass the array's name to a
// kernel: on the host it is only a stand-in, so its device address is looked
// up with cudaGetSymbolAddress, once per device, with that device current.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[JK_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mutex;
static void *g_noalloc_addr[JK_NOALLOC_MAX_DEVICES];

static int noalloc_scratch(int device, char **out)
{
    if (device < 0 || device >= JK_NOALLOC_MAX_DEVICES)
        return fail(JK_ERR_ARG, "jk_build_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[device]) {
        void *ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(JK_ERR_CUDA, std::string("jk_build_noalloc: cudaGetSymbolAddress: ") +
                                         cudaGetErrorString(e));
        g_noalloc_addr[device] = ptr;
    }
    *out = (char *)g_noalloc_addr[device];
    return JK_OK;
}

extern "C" int jk_build_noalloc(jk_plan *plan, const double *dm, int n_dm, int hermi, int with_j,
                                int with_k, double *vj, double *vk, double mixed_threshold,
                                void *stream)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_build_noalloc: plan is NULL");
    DeviceGuard g(plan->device);
    char *scratch = nullptr;
    const int rc = noalloc_scratch(plan->device, &scratch);
    if (rc) return rc;
    return build_one(plan, dm, n_dm, hermi, with_j, with_k, vj, vk, mixed_threshold,
                     (cudaStream_t)stream, scratch, (size_t)JK_NOALLOC_SCRATCH_BYTES, true,
                     "jk_build_noalloc");
}

extern "C" int jk_build_host(jk_plan *plan, const double *dm_host, int n_dm, int hermi, int with_j,
                             int with_k, double *vj_host, double *vk_host, double mixed_threshold,
                             void *stream)
{
    if (!plan || !dm_host) return fail(JK_ERR_ARG, "jk_build_host: null argument");
    if (n_dm <= 0) return fail(JK_ERR_ARG, "jk_build_host: no densities");
    DeviceGuard g(plan->device);
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)n_dm * plan->nao * plan->nao;
    const size_t need = 3 * n * sizeof(double);
    if (need > plan->io_size) {
        RC(engine_idle(plan->eng));
        cudaFree(plan->d_io);
        plan->d_io = nullptr;
        plan->io_size = 0;
        if (cudaMalloc(&plan->d_io, need) != cudaSuccess) {
            cudaGetLastError();
            return fail(JK_ERR_NOMEM, "jk_build_host: cannot allocate device buffers");
        }
        plan->io_size = need;
    }
    double *d_dm = plan->d_io, *d_vj = d_dm + n, *d_vk = d_vj + n;
    CK(cudaMemcpyAsync(d_dm, dm_host, n * sizeof(double), cudaMemcpyHostToDevice, st));
    RC(build_one(plan, d_dm, n_dm, hermi, with_j, with_k, with_j ? d_vj : nullptr,
                 with_k ? d_vk : nullptr, mixed_threshold, st, nullptr, 0, false, "jk_build_host"));
    if (with_j && vj_host)
        CK(cudaMemcpyAsync(vj_host, d_vj, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (with_k && vk_host)
        CK(cudaMemcpyAsync(vk_host, d_vk, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    return jk_sync(plan, stream);
}

extern "C" int jk_last_counts(jk_plan *plan, unsigned long long *quartets,
                              unsigned long long *prim_quartets,
                              unsigned long long *quartets_f32, int ncounts, int *nclasses)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_last_counts: plan is NULL");
    DeviceGuard g(plan->device);
    return engine_counts(plan->eng, quartets, prim_quartets, quartets_f32, ncounts, nclasses);
}

extern "C" int jk_set_timing(jk_plan *plan, int enable)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_set_timing: plan is NULL");
    DeviceGuard g(plan->device);
    return engine_set_timing(plan->eng, enable);
}

extern "C" int jk_last_class_ms(jk_plan *plan, float *ms, int ncounts, int *launches)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_last_class_ms: plan is NULL");
    DeviceGuard g(plan->device);
    return engine_class_ms(plan->eng, ms, ncounts, launches);
}

// ---------------------------------------------------------------------------
// batched builds over many plans
// ---------------------------------------------------------------------------
extern "C" int jk_batch_create(int device, jk_batch **out)
{
    if (!out) return fail(JK_ERR_ARG, "jk_batch_create: out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev ||
        device >= JK_MAX_DEVICES)
        return fail(JK_ERR_CUDA, "jk_batch_create: no CUDA device " + std::to_string(device));
    DeviceGuard g(device);
    jk_batch *b = new jk_batch();
    int rc = engine_init(b->eng, device);
    if (rc == JK_OK && cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking) != cudaSuccess)
        rc = fail(JK_ERR_CUDA, "jk_batch_create: cannot create the capture stream");
    if (rc != JK_OK) {
        engine_free(b->eng);
        delete b;
        return rc;
    }
    *out = b;
    return JK_OK;
}

extern "C" int jk_batch_destroy(jk_batch *batch)
{
    if (!batch) return JK_OK;
    DeviceGuard g(batch->eng.device);
    engine_idle(batch->eng);
    if (batch->gexec) cudaGraphExecDestroy(batch->gexec);
    if (batch->cap_stream) cudaStreamDestroy(batch->cap_stream);
    engine_free(batch->eng);
    delete batch;
    return JK_OK;
}

extern "C" int jk_batch_build(jk_batch *batch, jk_plan *const *plans, int nplans,
                              const double *const *dms, const int *n_dm, int hermi, int with_j,
                              int with_k, double *const *vj, double *const *vk,
                              double mixed_threshold, int use_graph, void *stream)
{
    if (!batch) return fail(JK_ERR_ARG, "jk_batch_build: batch is NULL");
    if (!plans || !dms || !n_dm || nplans <= 0)
        return fail(JK_ERR_ARG, "jk_batch_build: empty batch or NULL arrays");
    if ((with_j && !vj) || (with_k && !vk)) return fail(JK_ERR_ARG, "jk_batch_build: output is NULL");
    Engine &E = batch->eng;
    DeviceGuard g(E.device);
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<Item> items(nplans);
    for (int i = 0; i < nplans; ++i) {
        items[i].p = plans[i];
        items[i].dm = dms[i];
        items[i].n_dm = n_dm[i];
        items[i].vj = with_j ? vj[i] : nullptr;
        items[i].vk = with_k ? vk[i] : nullptr;
    }
    const Spec s = coulomb_spec(hermi, with_j, with_k, mixed_threshold);
    batch->last_replayed = batch->last_captured = 0;
    if (!use_graph || !batch->warmed) {
        RC(engine_build(E, items, s, st, nullptr, 0, false, "jk_batch_build"));
        batch->warmed = true;
        return JK_OK;
    }
    RC(engine_prepare(E, items, s, nullptr, 0, false, "jk_batch_build"));
    const int spec[4] = {hermi, with_j, with_k, E.shard_rank * 65536 + E.shard_size};
    const bool same = batch->gexec && E.blob == batch->graph_blob && E.blob_dev == batch->graph_blob &&
                      batch->graph_alloc_gen == E.alloc_gen && batch->graph_tune_gen == E.tune_gen &&
                      std::memcmp(spec, batch->graph_spec, sizeof(spec)) == 0 &&
                      batch->graph_mixed == mixed_threshold;
    RC(engine_upload(E, st));
    if (!same) {
        if (batch->gexec) {
            cudaGraphExecDestroy(batch->gexec);
            batch->gexec = nullptr;
        }
        RC(engine_configure(E));
        CK(cudaStreamBeginCapture(batch->cap_stream, cudaStreamCaptureModeRelaxed));
        const int rc = engine_launch(E, batch->cap_stream, false);
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(batch->cap_stream, &graph);
        if (rc != JK_OK) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        CK(ce);
        const cudaError_t ie = cudaGraphInstantiate(&batch->gexec, graph, 0);
        cudaGraphDestroy(graph);
        CK(ie);
        batch->graph_blob = E.blob;
        batch->graph_alloc_gen = E.alloc_gen;
        batch->graph_tune_gen = E.tune_gen;
        std::memcpy(batch->graph_spec, spec, sizeof(spec));
        batch->graph_mixed = mixed_threshold;
        batch->graph_launches = E.launches;
        batch->last_captured = 1;
    } else {
        batch->last_replayed = 1;
    }
    CK(cudaGraphLaunch(batch->gexec, st));
    E.launches = batch->graph_launches;
    if (E.timing) std::fill(E.ev_used.begin(), E.ev_used.end(), 0);
    return engine_finish(E, st);
}

extern "C" int jk_batch_sync(jk_batch *batch, void *stream)
{
    if (!batch) return fail(JK_ERR_ARG, "jk_batch_sync: batch is NULL");
    DeviceGuard g(batch->eng.device);
    return engine_sync(batch->eng, (cudaStream_t)stream, "jk_batch_sync");
}

extern "C" int jk_batch_counts(jk_batch *batch, unsigned long long *quartets,
                               unsigned long long *prim_quartets,
                               unsigned long long *quartets_f32, int ncounts, int *nclasses)
{
    if (!batch) return fail(JK_ERR_ARG, "jk_batch_counts: batch is NULL");
    DeviceGuard g(batch->eng.device);
    return engine_counts(batch->eng, quartets, prim_quartets, quartets_f32, ncounts, nclasses);
}

extern "C" int jk_batch_set_timing(jk_batch *batch, int enable)
{
    if (!batch) return fail(JK_ERR_ARG, "jk_batch_set_timing: batch is NULL");
    DeviceGuard g(batch->eng.device);
    return engine_set_timing(batch->eng, enable);
}

extern "C" int jk_batch_class_ms(jk_batch *batch, float *ms, int ncounts, int *launches)
{
    if (!batch) return fail(JK_ERR_ARG, "jk_batch_class_ms: batch is NULL");
    DeviceGuard g(batch->eng.device);
    return engine_class_ms(batch->eng, ms, ncounts, launches);
}

extern "C" int jk_batch_set_tuning(jk_batch *batch, int cls, int tasks_per_sm, int blocks_per_sm,
                                   int fp32)
{
    if (!batch) return fail(JK_ERR_ARG, "jk_batch_set_tuning: batch is NULL");
    return engine_set_tuning(batch->eng, cls, tasks_per_sm, blocks_per_sm, fp32);
}

extern "C" int jk_batch_stats(jk_batch *batch, int *graph_replayed, int *graph_captured,
                              long long *workspace_bytes)
{
    if (!batch) return fail(JK_ERR_ARG, "jk_batch_stats: batch is NULL");
    if (graph_replayed) *graph_replayed = batch->last_replayed;
    if (graph_captured) *graph_captured = batch->last_captured;
    if (workspace_bytes)
        *workspace_bytes = (long long)(batch->eng.ws_size + batch->eng.blob_cap +
                                       JK_CLASS_STREAMS * 4 * (size_t)batch->eng.max_rows *
                                           sizeof(int));
    return JK_OK;
}

// ---------------------------------------------------------------------------
// class table and measurement helpers
// ---------------------------------------------------------------------------
extern "C" int jk_class_info(int k, int *li, int *lj, int *lk, int *ll, int *form)
{
    if (k < 0 || k >= JK_NCLASSES) return fail(JK_ERR_ARG, "jk_class_info: no such class");
    const ClassEntry &c = jk_class_table[k];
    if (li) *li = c.li;
    if (lj) *lj = c.lj;
    if (lk) *lk = c.lk;
    if (ll) *ll = c.ll;
    if (form) *form = c.form;
    return JK_OK;
}

// FP64 FMA throughput probe: 8 independent chains per thread, all in registers
__global__ void fp64_fma_probe(double *out, int iters, double a, double b)
{
    double x0 = threadIdx.x * 1e-3, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
    double x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    const double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 12345.678) out[0] = s;   // keeps the chains live
}

extern "C" int jk_fp64_peak(int device, double *tflops)
{
    if (!tflops) return fail(JK_ERR_ARG, "jk_fp64_peak: tflops is NULL");
    DeviceGuard g(device);
    int nsm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    double *d_out = nullptr;
    CK(cudaMalloc(&d_out, sizeof(double)));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const int threads = 512, blocks = nsm * 4, iters = 4096;
    fp64_fma_probe<<<blocks, threads>>>(d_out, 64, 0.999999, 1e-7);   // warm-up
    CK(cudaGetLastError());
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        CK(cudaEventRecord(e0));
        fp64_fma_probe<<<blocks, threads>>>(d_out, iters, 0.999999, 1e-7);
        CK(cudaEventRecord(e1));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, ms);
    }
    const double flops = 2.0 * 16 * 8 * (double)iters * threads * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_out);
    return JK_OK;
}

extern "C" const char *jk_last_error(void) { return g_err.c_str(); }
