// Plan construction, build driver and C ABI of the B200 J/K engine
// (declared in include/jk_b200.h).
#include <algorithm>
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

struct jk_plan {
    int device = 0;
    int num_sms = 148;
    int nbas_user = 0, nbas = 0, nao = 0;
    bool expanded = false;          // a general contraction was split
    std::vector<int> sh_l, sh_ao, sh_user;
    double tol = 1e-13;
    float log_tol = 0.f;
    float q_max = -INFINITY, q_drop_max = -INFINITY;
    long long npairs = 0;
    int pc_off[NPAIR_CLASSES + 1] = {0};
    int pc_maxprim[NPAIR_CLASSES] = {0};
    std::vector<float> q_full;      // nbas x nbas (expanded numbering)
    // device tables
    ShellDev *d_shells = nullptr;
    double *d_basis = nullptr;
    double *d_prim = nullptr;
    PairRec *d_pairs = nullptr;
    double *d_rys = nullptr;
    float *d_rys32 = nullptr;
    int *d_sh_ao = nullptr, *d_sh_nf = nullptr;
    int *d_counters = nullptr;
    int *d_chunk = nullptr;         // task size per class of the last build
    unsigned long long *d_nq = nullptr;
    int *d_error = nullptr;
    float *d_dm_max = nullptr;
    // ket sub-lists (equal primitive-pair count) per pair class
    std::vector<int2> subs;
    int sub_off[NPAIR_CLASSES + 1] = {0};
    int2 *d_subs = nullptr;
    // task rows of one class launch: candidates, chunks, prefix of chunks
    int *d_rows = nullptr;
    long long max_rows = 0;
    void *d_cub = nullptr;
    size_t cub_bytes = 0;
    // workspace
    char *d_ws = nullptr;
    size_t ws_size = 0;
    double *d_io = nullptr;         // device buffers of jk_build_host
    size_t io_size = 0;
    cudaStream_t last_stream = nullptr;
    // per-class timing and launch count of the last build
    bool timing = false;
    std::vector<cudaEvent_t> ev;    // 2 per class
    std::vector<char> ev_used;
    int launches = 0;
};

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }
static int pair_class(int la, int lb) { return la * (la + 1) / 2 + lb; }

static double common_fac(int l)
{
    if (l == 0) return 0.282094791773878143;
    if (l == 1) return 0.488602511902919921;
    return 1.0;
}

static void free_plan(jk_plan *p)
{
    cudaFree(p->d_shells);
    cudaFree(p->d_basis);
    cudaFree(p->d_prim);
    cudaFree(p->d_pairs);
    cudaFree(p->d_rys);
    cudaFree(p->d_rys32);
    cudaFree(p->d_sh_ao);
    cudaFree(p->d_sh_nf);
    cudaFree(p->d_counters);
    cudaFree(p->d_nq);
    cudaFree(p->d_error);
    cudaFree(p->d_dm_max);
    cudaFree(p->d_ws);
    cudaFree(p->d_io);
    cudaFree(p->d_subs);
    cudaFree(p->d_rows);
    cudaFree(p->d_chunk);
    cudaFree(p->d_cub);
}

template <class T>
static cudaError_t upload(T **dst, const std::vector<T> &src)
{
    size_t bytes = std::max<size_t>(1, src.size()) * sizeof(T);
    cudaError_t e = cudaMalloc((void **)dst, bytes);
    if (e != cudaSuccess) return e;
    if (!src.empty()) e = cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
    return e;
}

static int plan_create(const int *atm, int natm, const int *bas, int nbas_user, const double *env,
                       const int *ao_loc, double tol, int device, jk_plan *p)
{
    if (!atm || !bas || !env || !ao_loc || natm <= 0 || nbas_user <= 0)
        return fail(JK_ERR_ARG, "jk_plan_create: null array or empty molecule");
    if (!(tol > 0.0)) return fail(JK_ERR_ARG, "jk_plan_create: direct_scf_tol must be > 0");
    p->device = device;
    p->tol = tol;
    p->log_tol = (float)std::log(tol);
    p->nbas_user = nbas_user;
    CK(cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, device));

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

    CK(upload(&p->d_shells, shells));
    CK(upload(&p->d_basis, basis));
    int4 *d_rec = nullptr, *d_cand = nullptr;
    float *d_q = nullptr;
    CK(upload(&d_rec, rec));
    CK(upload(&d_cand, cand));
    CK(cudaMalloc(&p->d_prim, std::max<size_t>(1, rec.size()) * JK_PRIM_STRIDE * sizeof(double)));
    CK(cudaMalloc(&d_q, std::max<size_t>(1, cand.size()) * sizeof(float)));

    std::vector<double> rys_host(RYS_TOTAL);
    std::memcpy(rys_host.data(), rys_table_host, sizeof(rys_table_host));
    std::vector<float> rys32_host(RYS32_TOTAL);
    std::memcpy(rys32_host.data(), rys_table32_host, sizeof(rys_table32_host));
    for (int n = 0; n < RYS_NMAX; ++n)
        for (int k = 0; k < RYS_NMAX; ++k) {
            rys_host[RYS_LARGEX_OFF + n * RYS_NMAX + k] = rys_largex_r_host[n][k];
            rys_host[RYS_LARGEX_OFF + RYS_NMAX * RYS_NMAX + n * RYS_NMAX + k] = rys_largex_w_host[n][k];
            rys32_host[RYS32_LARGEX_OFF + n * RYS_NMAX + k] = (float)rys_largex_r_host[n][k];
            rys32_host[RYS32_LARGEX_OFF + RYS_NMAX * RYS_NMAX + n * RYS_NMAX + k] =
                (float)rys_largex_w_host[n][k];
        }
    CK(upload(&p->d_rys, rys_host));
    CK(upload(&p->d_rys32, rys32_host));

    if (!rec.empty()) {
        const int nt = 256;
        prim_pair_fill_kernel<<<(unsigned)((rec.size() + nt - 1) / nt), nt>>>(
            d_rec, (long long)rec.size(), p->d_shells, p->d_basis, p->d_prim);
        CK(cudaGetLastError());
        schwarz_kernel<<<(unsigned)((cand.size() + 127) / 128), 128>>>(
            d_cand, (int)cand.size(), p->d_shells, p->d_prim, p->d_rys, d_q);
        CK(cudaGetLastError());
    }
    std::vector<float> q(cand.size());
    if (!cand.empty()) CK(cudaMemcpy(q.data(), d_q, q.size() * sizeof(float), cudaMemcpyDeviceToHost));
    cudaFree(d_rec);
    cudaFree(d_cand);
    cudaFree(d_q);

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
    for (int k = 0; k < NPAIR_CLASSES; ++k) {
        auto &v = byclass[k];
        // primitive-pair count first (sub-lists of equal loop bounds), then q
        std::stable_sort(v.begin(), v.end(), [&](int a, int b) {
            if (cand[a].w != cand[b].w) return cand[a].w > cand[b].w;
            return q[a] > q[b];
        });
        p->pc_off[k] = (int)recs.size();
        p->sub_off[k] = (int)p->subs.size();
        for (size_t t = 0; t < v.size(); ++t) {
            if (t == 0 || cand[v[t]].w != cand[v[t - 1]].w)
                p->subs.push_back(make_int2((int)t, (int)t));
            p->subs.back().y = (int)t + 1;
        }
        int mp = 0;
        for (int c : v) {
            const int i = cand[c].x, j = cand[c].y;
            PairRec r;
            r.ish = i;
            r.jsh = j;
            r.i0 = p->sh_ao[i];
            r.j0 = p->sh_ao[j];
            r.prim0 = cand[c].z;
            r.nprim = cand[c].w;
            r.q = q[c];
            r.pad = 0.f;
            r.ABx = shells[i].x - shells[j].x;
            r.ABy = shells[i].y - shells[j].y;
            r.ABz = shells[i].z - shells[j].z;
            mp = std::max(mp, r.nprim);
            recs.push_back(r);
        }
        p->pc_maxprim[k] = mp;
    }
    p->pc_off[NPAIR_CLASSES] = (int)recs.size();
    p->sub_off[NPAIR_CLASSES] = (int)p->subs.size();
    CK(upload(&p->d_subs, p->subs));
    // task rows: the largest (bra class pairs) x (ket class sub-lists)
    long long max_rows = 1;
    for (int A = 0; A < NPAIR_CLASSES; ++A)
        for (int B = 0; B <= A; ++B)
            max_rows = std::max<long long>(
                max_rows, (long long)(p->pc_off[A + 1] - p->pc_off[A]) *
                              (p->sub_off[B + 1] - p->sub_off[B]));
    if (max_rows > (1ll << 31) - 1) return fail(JK_ERR_ARG, "molecule too large (task rows)");
    CK(cudaMalloc(&p->d_rows, 4 * (size_t)max_rows * sizeof(int)));
    CK(cudaMalloc(&p->d_chunk, JK_NCLASSES * sizeof(int)));
    p->max_rows = max_rows;
    p->cub_bytes = 0;
    CK(cub::DeviceScan::InclusiveSum(nullptr, p->cub_bytes, p->d_rows, p->d_rows, (int)max_rows));
    CK(cudaMalloc(&p->d_cub, std::max<size_t>(16, p->cub_bytes)));
    p->npairs = (long long)recs.size();
    CK(upload(&p->d_pairs, recs));

    std::vector<int> nf(nbas);
    for (int s = 0; s < nbas; ++s) nf[s] = ncart(shells[s].l);
    CK(upload(&p->d_sh_ao, p->sh_ao));
    CK(upload(&p->d_sh_nf, nf));
    CK(cudaMalloc(&p->d_counters, JK_NCLASSES * sizeof(int)));
    CK(cudaMalloc(&p->d_nq, 3 * JK_NCLASSES * sizeof(unsigned long long)));
    CK(cudaMalloc(&p->d_error, sizeof(int)));
    CK(cudaMemset(p->d_error, 0, sizeof(int)));
    CK(cudaMemset(p->d_nq, 0, 3 * JK_NCLASSES * sizeof(unsigned long long)));
    CK(cudaMalloc(&p->d_dm_max, sizeof(float)));
    CK(cudaDeviceSynchronize());
    return JK_OK;
}

extern "C" int jk_plan_create(const int *atm, int natm, const int *bas, int nbas, const double *env,
                              const int *ao_loc, double direct_scf_tol, int device, jk_plan **out)
{
    if (!out) return fail(JK_ERR_ARG, "jk_plan_create: out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
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
    cudaDeviceSynchronize();
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

extern "C" int jk_plan_q_cond(const jk_plan *plan, float *q_host, int nbas)
{
    if (!plan || !q_host) return fail(JK_ERR_ARG, "jk_plan_q_cond: null argument");
    if (plan->expanded || nbas != plan->nbas)
        return fail(JK_ERR_ARG, "jk_plan_q_cond: nbas does not match the plan's shells");
    std::memcpy(q_host, plan->q_full.data(), plan->q_full.size() * sizeof(float));
    return JK_OK;
}

static size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

// ws_ext: when not NULL, the build's workspace is taken from this caller-owned
// device buffer of ws_ext_size bytes instead of the plan's own allocation.
static int build_impl(jk_plan *p, const double *dm, int n_dm, int hermi, int with_j, int with_k,
                      double *vj, double *vk, double mixed_threshold, cudaStream_t st,
                      char *ws_ext = nullptr, size_t ws_ext_size = 0)
{
    if (n_dm <= 0 || !dm) return fail(JK_ERR_ARG, "jk_build: no densities");
    if (hermi < 0 || hermi > 2) return fail(JK_ERR_ARG, "jk_build: hermi must be 0, 1 or 2");
    if ((with_j && !vj) || (with_k && !vk)) return fail(JK_ERR_ARG, "jk_build: output is NULL");
    const float log_mixed = mixed_threshold > 0 ? (float)std::log(mixed_threshold) : -INFINITY;
    const int nao = p->nao;
    const size_t nao2 = (size_t)nao * nao;
    const int n_k = with_k ? (hermi == 0 ? 2 * n_dm : n_dm) : 0;
    const int n_j = (with_j && hermi != 2) ? n_dm : 0;
    const bool need_t = with_k && hermi == 0;
    // workspace: Kh | Jh | dsJ | DT | dm_cond
    const size_t o_kh = 0;
    const size_t o_jh = o_kh + align256((size_t)n_k * nao2 * 8);
    const size_t o_ds = o_jh + align256((size_t)n_j * nao2 * 8);
    const size_t o_dt = o_ds + align256((size_t)n_j * nao2 * 8);
    const size_t o_dc = o_dt + align256(need_t ? (size_t)n_dm * nao2 * 8 : 0);
    const size_t need = o_dc + align256((size_t)p->nbas * p->nbas * 4);
    char *ws = p->d_ws;
    if (ws_ext) {
        if (need > ws_ext_size)
            return fail(JK_ERR_RANGE, "jk_build_noalloc: this build needs " + std::to_string(need) +
                                          " bytes of scratch, the library's static scratch holds " +
                                          std::to_string(ws_ext_size) +
                                          " (use jk_build for larger molecules or more densities)");
        ws = ws_ext;
    } else if (need > p->ws_size) {
        CK(cudaStreamSynchronize(st));
        cudaFree(p->d_ws);
        p->d_ws = nullptr;
        p->ws_size = 0;
        if (cudaMalloc(&p->d_ws, need) != cudaSuccess) {
            cudaGetLastError();
            return fail(JK_ERR_NOMEM, "jk_build: cannot allocate " + std::to_string(need) +
                                          " bytes of workspace");
        }
        p->ws_size = need;
        ws = p->d_ws;
    }
    double *Kh = (double *)(ws + o_kh);
    double *Jh = (double *)(ws + o_jh);
    double *dsJ = (double *)(ws + o_ds);
    double *DT = (double *)(ws + o_dt);
    float *dmc = (float *)(ws + o_dc);
    p->last_stream = st;
    p->launches = 0;
    if (p->timing) std::fill(p->ev_used.begin(), p->ev_used.end(), 0);

    const dim3 tb(32, 8);
    const dim3 tg((nao + 31) / 32, (nao + 31) / 32, n_dm);
    if (n_j) {
        add_transpose_kernel<<<tg, tb, 0, st>>>(dm, dm, 1.0, nao, dsJ);
        CK(cudaGetLastError());
        p->launches++;
        CK(cudaMemsetAsync(Jh, 0, (size_t)n_j * nao2 * 8, st));
    }
    if (need_t) {
        transpose_kernel<<<tg, tb, 0, st>>>(dm, nao, DT);
        CK(cudaGetLastError());
        p->launches++;
    }
    if (n_k) CK(cudaMemsetAsync(Kh, 0, (size_t)n_k * nao2 * 8, st));
    {
        const dim3 b2(16, 16);
        const dim3 g2((p->nbas + 15) / 16, (p->nbas + 15) / 16);
        dm_cond_kernel<<<g2, b2, 0, st>>>(dm, n_dm, nao, p->d_sh_ao, p->d_sh_nf, p->nbas, dmc);
        CK(cudaGetLastError());
        max_reduce_kernel<<<1, 1024, 0, st>>>(dmc, (long long)p->nbas * p->nbas, p->d_dm_max);
        CK(cudaGetLastError());
        range_check_kernel<<<1, 1, 0, st>>>(p->d_dm_max, p->q_drop_max, p->q_max, p->log_tol,
                                           p->d_error);
        CK(cudaGetLastError());
        p->launches += 3;
    }
    CK(cudaMemsetAsync(p->d_counters, 0, JK_NCLASSES * sizeof(int), st));
    CK(cudaMemsetAsync(p->d_nq, 0, 3 * JK_NCLASSES * sizeof(unsigned long long), st));

    if (n_j || n_k) {
        LaunchCfg cfg;
        cfg.stream = st;
        cfg.num_sms = p->num_sms;
        cfg.blocks_per_sm = 0;
        cfg.mixed = 0;
        char launch_msg[256] = {0};
        cfg.msg = launch_msg;
        for (int c = 0; c < JK_NCLASSES; ++c) {
            const ClassEntry &ce = jk_class_table[c];
            const int A = ce.bra_class, B = ce.ket_class;
            const int nbra = p->pc_off[A + 1] - p->pc_off[A];
            const int nket = p->pc_off[B + 1] - p->pc_off[B];
            if (nbra == 0 || nket == 0) continue;
            ClassArgs a;
            a.bra = p->d_pairs + p->pc_off[A];
            a.ket = p->d_pairs + p->pc_off[B];
            a.nbra = nbra;
            a.nket = nket;
            a.same_class = A == B;
            a.max_bra_prim = p->pc_maxprim[A];
            a.prim = p->d_prim;
            a.rys = p->d_rys;
            a.rys32 = p->d_rys32;
            a.dm_cond = dmc;
            a.nbas = p->nbas;
            a.log_tol = p->log_tol;
            a.dm_max = p->d_dm_max;
            a.nao = nao;
            a.dmK = dm;
            a.dmKT = DT;
            a.n_ka = n_k ? n_dm : 0;
            a.n_k = n_k;
            a.dsJ = dsJ;
            a.n_j = n_j;
            a.Kh = Kh;
            a.Jh = Jh;
            a.counter = p->d_counters + c;
            a.sub = p->d_subs + p->sub_off[B];
            a.nsub = p->sub_off[B + 1] - p->sub_off[B];
            a.chunk = p->d_chunk + c;
            a.row_ncand = p->d_rows;
            int *chunks = p->d_rows + p->max_rows;
            int *prefix = p->d_rows + 2 * p->max_rows;
            int *cand_prefix = p->d_rows + 3 * p->max_rows;
            a.row_prefix = prefix;
            const int rows = nbra * a.nsub;
            a.nquartets = p->d_nq + c;
            a.nprimq = p->d_nq + JK_NCLASSES + c;
            a.mixed_log_thr = log_mixed;
            a.nquartets32 = p->d_nq + 2 * JK_NCLASSES + c;
            a.error = p->d_error;
            if (p->timing) CK(cudaEventRecord(p->ev[2 * c], st));
            // task list: candidates per row, a chunk size giving ~16 tasks per
            // SM, chunks per row, prefix sum of chunks
            task_rows_kernel<<<(rows + 255) / 256, 256, 0, st>>>(a);
            CK(cudaGetLastError());
            size_t tmp_bytes = p->cub_bytes;
            CK(cub::DeviceScan::InclusiveSum(p->d_cub, tmp_bytes, p->d_rows, cand_prefix, rows, st));
            const int lo = ce.form == 0 ? 128 : 32, hi = ce.form == 0 ? 4096 : 1024;
            const int target = (ce.form == 0 ? 64 : 16) * p->num_sms;
            task_chunks_kernel<<<(rows + 255) / 256, 256, 0, st>>>(
                p->d_rows, cand_prefix, rows, target, lo, hi, p->d_chunk + c, chunks);
            CK(cudaGetLastError());
            tmp_bytes = p->cub_bytes;
            CK(cub::DeviceScan::InclusiveSum(p->d_cub, tmp_bytes, chunks, prefix, rows, st));
            p->launches += 4;
            int rc = ce.launch(a, cfg);
            if (rc != 0)
                return fail(JK_ERR_CUDA, std::string("class kernel launch failed: ") + launch_msg + " " +
                                             cudaGetErrorString((cudaError_t)rc));
            if (p->timing) {
                CK(cudaEventRecord(p->ev[2 * c + 1], st));
                p->ev_used[c] = 1;
            }
            p->launches++;
        }
    }
    // assemble J and K
    if (with_j) {
        if (n_j) {
            add_transpose_kernel<<<tg, tb, 0, st>>>(Jh, Jh, 1.0, nao, vj);
            CK(cudaGetLastError());
            p->launches++;
        } else {
            CK(cudaMemsetAsync(vj, 0, (size_t)n_dm * nao2 * 8, st));
        }
    }
    if (with_k) {
        if (hermi == 0)
            add_transpose_kernel<<<tg, tb, 0, st>>>(Kh, Kh + (size_t)n_dm * nao2, 1.0, nao, vk);
        else
            add_transpose_kernel<<<tg, tb, 0, st>>>(Kh, Kh, hermi == 2 ? -1.0 : 1.0, nao, vk);
        CK(cudaGetLastError());
        p->launches++;
    }
    return JK_OK;
}

extern "C" int jk_build(jk_plan *plan, const double *dm, int n_dm, int hermi, int with_j,
                        int with_k, double *vj, double *vk, double mixed_threshold, void *stream)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_build: plan is NULL");
    DeviceGuard g(plan->device);
    return build_impl(plan, dm, n_dm, hermi, with_j, with_k, vj, vk, mixed_threshold,
                      (cudaStream_t)stream);
}

extern "C" int jk_sync(jk_plan *plan, void *stream)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_sync: plan is NULL");
    DeviceGuard g(plan->device);
    CK(cudaStreamSynchronize((cudaStream_t)stream));
    int err = 0;
    CK(cudaMemcpy(&err, plan->d_error, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
        CK(cudaMemset(plan->d_error, 0, sizeof(int)));
        if (err == JK_ERR_RANGE)
            return fail(JK_ERR_RANGE, "density elements exceed the range the plan was built for "
                                      "(shell pairs it dropped would pass the screening)");
        return fail(JK_ERR_DEVICE, "kernel error flag " + std::to_string(err));
    }
    return JK_OK;
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
    return build_impl(plan, dm, n_dm, hermi, with_j, with_k, vj, vk, mixed_threshold,
                      (cudaStream_t)stream, scratch, (size_t)JK_NOALLOC_SCRATCH_BYTES);
}

extern "C" int jk_build_host(jk_plan *plan, const double *dm_host, int n_dm, int hermi, int with_j,
                             int with_k, double *vj_host, double *vk_host, double mixed_threshold,
                             void *stream)
{
    if (!plan || !dm_host) return fail(JK_ERR_ARG, "jk_build_host: null argument");
    DeviceGuard g(plan->device);
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)n_dm * plan->nao * plan->nao;
    const size_t need = 3 * n * sizeof(double);
    if (need > plan->io_size) {
        CK(cudaStreamSynchronize(st));
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
    int rc = build_impl(plan, d_dm, n_dm, hermi, with_j, with_k, with_j ? d_vj : nullptr,
                        with_k ? d_vk : nullptr, mixed_threshold, st);
    if (rc) return rc;
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
    if (nclasses) *nclasses = JK_NCLASSES;
    if (!quartets && !prim_quartets && !quartets_f32) return JK_OK;
    DeviceGuard g(plan->device);
    CK(cudaStreamSynchronize(plan->last_stream));
    std::vector<unsigned long long> h(3 * JK_NCLASSES);
    CK(cudaMemcpy(h.data(), plan->d_nq, 3 * JK_NCLASSES * sizeof(unsigned long long),
                  cudaMemcpyDeviceToHost));
    for (int k = 0; k < ncounts && k < JK_NCLASSES; ++k) {
        if (quartets) quartets[k] = h[k];
        if (prim_quartets) prim_quartets[k] = h[JK_NCLASSES + k];
        if (quartets_f32) quartets_f32[k] = h[2 * JK_NCLASSES + k];
    }
    return JK_OK;
}

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

extern "C" int jk_set_timing(jk_plan *plan, int enable)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_set_timing: plan is NULL");
    DeviceGuard g(plan->device);
    if (enable && plan->ev.empty()) {
        plan->ev.resize(2 * JK_NCLASSES);
        for (auto &e : plan->ev) CK(cudaEventCreate(&e));
        plan->ev_used.assign(JK_NCLASSES, 0);
    }
    plan->timing = enable != 0;
    return JK_OK;
}

extern "C" int jk_last_class_ms(jk_plan *plan, float *ms, int ncounts, int *launches)
{
    if (!plan) return fail(JK_ERR_ARG, "jk_last_class_ms: plan is NULL");
    DeviceGuard g(plan->device);
    if (launches) *launches = plan->launches;
    if (!ms) return JK_OK;
    CK(cudaStreamSynchronize(plan->last_stream));
    for (int c = 0; c < ncounts && c < JK_NCLASSES; ++c) {
        ms[c] = 0.f;
        if (plan->timing && c < (int)plan->ev_used.size() && plan->ev_used[c])
            CK(cudaEventElapsedTime(&ms[c], plan->ev[2 * c], plan->ev[2 * c + 1]));
    }
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
