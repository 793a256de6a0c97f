/*
 * C ABI of the B200 direct-SCF Coulomb/exchange (J/K) engine,
 * libjk_b200.so.
 *
 * Every entry point returns 0 on success and a non-zero JK_ERR_* code
 * otherwise; jk_last_error() gives the message of the last failure on the
 * calling thread.  There is no fallback path: a shell the engine cannot
 * handle (l > 3) or a density out of the plan's range is an error.
 *
 * Conventions
 *   - Molecules are passed in PySCF's integer/float layout: atm[natm][6],
 *     bas[nbas][8], env[] (the arrays of a pyscf.gto.Mole: _atm, _bas,
 *     _env).  Contraction coefficients in env carry PySCF's radial
 *     normalisation; the s/p angular factor of libcint is applied here.
 *   - Densities and results are row-major (n, nao, nao) float64 arrays in
 *     the Cartesian AO basis, AO order given by ao_loc (PySCF's
 *     mol.ao_loc_nr(cart=True)); general contractions are expanded
 *     contraction-major, as PySCF orders them.
 *   - vj[k,l] = sum_ij (ij|kl) D[j,i],  vk[i,l] = sum_jk (ij|kl) D[j,k]
 *     (PySCF's dot_eri_dm conventions).  hermi = 1: D symmetric; hermi = 2:
 *     D antisymmetric (vj is zero); hermi = 0: no symmetry.
 *   - Device pointers unless a name says _host.  Calls are asynchronous on
 *     the given stream (NULL: the default stream); jk_sync() waits and
 *     returns a device-side error, if any.
 *   - One plan per stream at a time; a plan reuses its device workspace
 *     across calls (one SCF cycle after another).
 */
#ifndef JK_B200_H
#define JK_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define JK_OK 0
#define JK_ERR_ARG 1          /* invalid argument                         */
#define JK_ERR_UNSUPPORTED 2  /* shell type the engine does not handle     */
#define JK_ERR_CUDA 3         /* CUDA runtime error                        */
#define JK_ERR_NOMEM 4        /* device allocation failed                  */
#define JK_ERR_RANGE 5        /* density beyond the plan's screening range */
#define JK_ERR_DEVICE 6       /* error flag raised inside a kernel         */
#define JK_ERR_SCRATCH 7      /* jk_build_noalloc: the build needs more scratch
                                 than the library's fixed array (or the plan's
                                 reservation) holds; jk_build can run it     */

typedef struct jk_plan jk_plan;

/*
 * Build a plan: shell-pair and primitive-pair tables, Schwarz bounds
 * q_ij = log sqrt(max |(ij|ij)|), pair lists by angular-momentum class
 * sorted by q.  direct_scf_tol is the screening threshold of every later
 * build (PySCF's mol.direct_scf_tol; quartets are kept when
 * q_ij + q_kl + log max|D_block| > log(tol)).  device: CUDA ordinal.
 *
 * Replaces the plan GPU4PySCF's _VHFOpt.build() prepares and the
 * reference's per-call screening prep: electrolites/fastk.py:336-351 (_prep),
 * electrolites/compat.py:54-78 (dense_q_cond) and :84-149
 * (tril_pair_mappings).
 */
int jk_plan_create(const int *atm, int natm, const int *bas, int nbas,
                   const double *env, const int *ao_loc,
                   double direct_scf_tol, int device, jk_plan **out);

int jk_plan_destroy(jk_plan *plan);

/* nao (Cartesian) and the number of shell pairs kept by the plan. */
int jk_plan_info(const jk_plan *plan, int *nao, long long *npairs);

/*
 * J and/or K for n_dm densities dm[n_dm][nao][nao] (device).  vj and vk
 * (device, [n_dm][nao][nao]) are overwritten; either may be NULL when
 * with_j / with_k is 0.  mixed_threshold <= 0 gives the plain all-FP64
 * build; > 0 runs quartets whose screened bound
 * |(ij|ij)|^1/2 |(kl|kl)|^1/2 max|D| is below it with FP32 Rys evaluation
 * (FP64 accumulation).
 *
 * Replaces _VHFOpt.get_jk / get_k and j_engine._VHFOpt.get_j as the
 * reference patches them: electrolites/fastjk.py:276-357 (get_jk),
 * electrolites/fastk.py:642-741 (get_k), electrolites/fastj.py:540-569
 * (get_j_181), including their hermi post-processing.
 */
int jk_build(jk_plan *plan, const double *dm, int n_dm, int hermi,
             int with_j, int with_k, double *vj, double *vk,
             double mixed_threshold, void *stream);

/*
 * jk_build for the long-range operator erf(omega r)/r (omega > 0; omega = 0
 * is jk_build).  Replaces the reference's long-range path of
 * _VHFOpt.get_k (electrolites/fastk.py:642-741; the operator enters its
 * kernels as rsqrt(a_ij + a_kl + a_ij a_kl / omega^2),
 * electrolites/kernels/fastk_prologue.cu:281-288).
 */
int jk_build_rs(jk_plan *plan, const double *dm, int n_dm, int hermi,
                int with_j, int with_k, double *vj, double *vk,
                double mixed_threshold, double omega, void *stream);

/*
 * jk_build for the operator sum_t coef[t] * op(omega[t]) over n_terms (1 or
 * 2) terms, op(0) = 1/r and op(w > 0) = erf(w r)/r, in one pass over the
 * shell quartets: each primitive quartet evaluates the Rys quadrature once
 * per term, and screening, primitive data and the density contraction are
 * shared.  Range-separated exchange lr K_erf + sr K_erfc is
 * {sr, lr - sr} at {0, omega} (erfc(w r)/r = 1/r - erf(w r)/r).
 * Quartets are screened by their Coulomb bound, without the coefficients.
 * Replaces the reference's fused two-range K, get_k_rsh
 * (electrolites/fastk.py:774-899: coef_f K_full + coef_l K_lr in a single
 * pass, screened with the full-range q_cond); here J takes the same operator
 * when with_j is set.  Errors: n_terms outside 1..2, a negative or
 * non-finite omega, a non-finite coefficient.
 */
int jk_build_op(jk_plan *plan, const double *dm, int n_dm, int hermi,
                int with_j, int with_k, double *vj, double *vk,
                double mixed_threshold, int n_terms, const double *coef,
                const double *omega, void *stream);

/*
 * The same with host buffers: copies dm in, builds, copies vj/vk out, and
 * synchronises.  The call a CPU-side caller (PySCF's own get_jk) makes.
 */
int jk_build_host(jk_plan *plan, const double *dm_host, int n_dm, int hermi,
                  int with_j, int with_k, double *vj_host, double *vk_host,
                  double mixed_threshold, void *stream);

/*
 * jk_build without any device allocation.  No counterpart in the reference:
 * it exists for callers that cannot let a library call cudaMalloc -- an SCF
 * driver that hands all device memory to its own caching pool (PyTorch,
 * CuPy) and would fragment it or run out behind the pool's back, a
 * latency-critical serving path where a cudaMalloc or cudaFree would
 * synchronise the device, or a host that only allows memory it manages.
 *
 * The build's scratch (half-J/K accumulators, symmetrised and transposed
 * densities, density screening table) comes from one fixed array of
 * JK_NOALLOC_SCRATCH_BYTES inside the library, which every GPU that loads
 * the library keeps until the process exits.  A build whose scratch would
 * not fit -- about n_k + 2 n_j density-sized double matrices plus
 * nbas^2 floats, e.g. nao up to ~700 for two symmetric densities -- is
 * rejected with JK_ERR_SCRATCH before anything is launched.  The plan must
 * already exist (jk_plan_create allocates; create it at set-up); its
 * create-time reservations cover its own builds, so jk_build_noalloc may be
 * a plan's first build.
 *
 * The first call on a device looks up the array's device address (with
 * that device current).  The call is not capture-safe: it may wait on the
 * plan's previous build and reuses a pinned staging buffer, so it must not
 * be issued on a stream that is being captured into a CUDA graph (use
 * jk_batch_* with use_graph = 1 for graph replay).
 * Every call shares the one array and it keeps the previous call's
 * contents (the accumulators are cleared at the start of each call), so
 * calls whose work overlaps on the GPU -- different streams, or different
 * plans on one device -- race with each other: serialise them.
 */
#define JK_NOALLOC_SCRATCH_BYTES (24u << 20)
#define JK_NOALLOC_MAX_DEVICES 64
int jk_build_noalloc(jk_plan *plan, const double *dm, int n_dm, int hermi,
                     int with_j, int with_k, double *vj, double *vk,
                     double mixed_threshold, void *stream);

/*
 * Nuclear gradient of the two-electron energy: grad[natm][3] (device,
 * overwritten) = dE/dR_A of
 *     E = j_factor/2 Tr[Dt J[Dt]] - k_factor c sum_s Tr[D_s K[D_s]],
 * Dt = sum_s D_s, c = 1/4 for n_dm = 1 (a closed-shell total density) and
 * 1/2 for n_dm = 2 (the two spin densities), for the symmetric densities
 * dm[n_dm][nao][nao] (device) held fixed in the AO basis while the atoms
 * and their basis functions move.  omega > 0 takes the long-range operator
 * erf(omega r)/r.  Quartets are screened as by jk_build (Coulomb and
 * exchange tests together).
 *
 * Replaces GPU4PySCF's _jk_energy_per_atom as the reference patches it
 * (electrolites/fastejk.py:276-356, the factors at :308-316;
 * electrolites/codegen/gen_ejk.py:102-144 for its kernels).
 */
int jk_grad(jk_plan *plan, const double *dm, int n_dm, double j_factor,
            double k_factor, double omega, double *grad, void *stream);

/* Wait for the plan's work on stream; returns JK_ERR_DEVICE if a kernel
 * raised its error flag (the flag is then cleared). */
int jk_sync(jk_plan *plan, void *stream);

/*
 * Shell quartets, primitive quartets and FP32-evaluated quartets of the
 * last build, per angular-momentum class (index k of jk_class_info), and
 * the number of classes.  Any array may be NULL.  Synchronises the stream
 * of the last build.
 */
int jk_last_counts(jk_plan *plan, unsigned long long *quartets,
                   unsigned long long *prim_quartets,
                   unsigned long long *quartets_f32, int ncounts,
                   int *nclasses);

/* li, lj, lk, ll and the form (0 register, 1 team) of class k. */
int jk_class_info(int k, int *li, int *lj, int *lk, int *ll, int *form);

/*
 * Per-class kernel timing.  enable = 1: every later build records CUDA
 * events around each class kernel and runs all class kernels on the build's
 * stream (otherwise they are spread over two streams to overlap their
 * tails), so each class is timed alone; enable = 2: the class kernels keep
 * their two streams and each class's events are recorded on its own stream
 * (the class times of the default launch order, overlap included);
 * enable = 0: no events.
 * jk_last_class_ms() then returns the milliseconds of each class kernel of
 * the last build (0 for classes not launched) and the number of kernels the
 * library launched in that build.  Synchronises the last build's stream.
 */
int jk_set_timing(jk_plan *plan, int enable);
int jk_last_class_ms(jk_plan *plan, float *ms, int ncounts, int *launches);

/*
 * Measurement helper, no counterpart in the reference: the FP64 FMA
 * throughput of the device (TFLOP/s, 2 flops per FMA) from a
 * register-resident FMA chain on every SM, timed with CUDA events.
 */
int jk_fp64_peak(int device, double *tflops);

/* Schwarz bounds q[nbas][nbas] (host, float, -inf for pairs below the
 * plan's range), in the caller's shell numbering when no shell has a
 * general contraction. */
int jk_plan_q_cond(const jk_plan *plan, float *q_host, int nbas);

/* Device memory the plan holds: its pair tables and task-row buffers, and
 * the workspace of its own builds (grown on demand and kept). */
int jk_plan_memory(const jk_plan *plan, long long *table_bytes,
                   long long *workspace_bytes);

/*
 * Multi-GPU sharding of a plan's builds: with size > 1 a build evaluates
 * only the tasks t = rank + size * n of every class's task list, so the
 * vj / vk it returns are this rank's part and the sum over ranks (an
 * all-reduce) is the full result.  All ranks must build with the same
 * plan parameters and densities.  size = 1 (the default) is the whole build.
 * No counterpart in the reference, which runs on one GPU
 * (electrolites/fastk.py:657).
 */
int jk_plan_set_shard(jk_plan *plan, int rank, int size);

/*
 * Screening threshold of the plan's later builds (single and batched):
 * quartets are kept when q_ij + q_kl + log max|D| > log(tol).  tol must be
 * at least the plan's direct_scf_tol (its pair lists hold only the pairs
 * that threshold can need); tol equal to it restores the default.  The
 * counterpart of raising _VHFOpt.direct_scf_tol between builds, which the
 * reference's loose-then-tight SCF screening does for its loose cycles
 * (electrolites/fastscfscreen.py:107-118; the builds read the attribute at
 * call time).
 */
int jk_plan_set_tol(jk_plan *plan, double tol);

/*
 * J engine of the plan's builds (on by default): J of every quartet from its
 * (e0|f0) block contracted with the pairs'
 * x-space densities D~ = H^T (D + D^T) (H: a pair's horizontal transfer)
 * instead of the (ij|kl) digest (K, if asked for, still from (ij|kl)); the
 * x-space J of every pair is transferred back once per build.  Same quartets, same
 * screening, same result to rounding; off (on = 0), J is digested from
 * (ij|kl).  The counterpart of the reference's J engine
 * for J-only builds, j_engine._VHFOpt.get_j (electrolites/fastj.py:540-569,
 * McMurchie-Davidson over Hermite densities; here the density contraction
 * happens in the Rys transfer's source space).  Batched and jk_build_noalloc
 * builds use the (ij|kl) digest.
 */
int jk_plan_set_jengine(jk_plan *plan, int on);

/*
 * Per-class launch tuning of the plan's builds: the number of tasks per SM
 * the task size aims at, a cap on resident blocks per SM (0: the occupancy
 * limit), and whether mixed-precision builds may run this class's
 * low-bound quartets in FP32 (1 yes, 0 no: FP64 throughout, -1 the class's
 * default).  cls = -1 restores the defaults of every class; a 0
 * tasks_per_sm restores that class's default.  Set by the autotuner
 * (electrolites_b200/autotune.py), which keeps FP32 only for the classes
 * where it measures faster; the reference picks its launch shapes in its
 * code generator (electrolites/codegen/gen_khigh.py).
 */
int jk_plan_set_tuning(jk_plan *plan, int cls, int tasks_per_sm, int blocks_per_sm,
                       int fp32);

/*
 * J-only builds: which classes take the McMurchie-Davidson J kernel in place
 * of the Rys J engine -- the reference's J engine
 * (electrolites/fastj.py:540-569, per-class kernels j_<lij>_<lkl>), here a
 * register-form kernel per class up to l_i + l_j + l_k + l_l = 6, chosen per
 * class by measurement.  mode 1: on, 0: off, -1: the class's default; cls =
 * -1: every class that has the kernel.  It serves builds of the Coulomb
 * operator with up to two densities; others keep the Rys J engine.
 * JK_ERR_ARG for a class without the kernel.
 */
int jk_plan_set_jmd(jk_plan *plan, int cls, int mode);

/*
 * Batched builds: J/K for many molecules (plans) in one launch stream, each
 * with its own densities (n_dm[i] of them, dms[i] on the device) and
 * outputs (vj[i], vk[i]).  Each angular-momentum class runs as one
 * persistent kernel over the task lists of every plan in the batch.
 * hermi, with_j, with_k and mixed_threshold apply to every plan and mean
 * what they mean for jk_build; the results equal those of one jk_build per
 * plan.  Arrays of pointers are host arrays.
 *
 * use_graph = 1: the launch stream is captured in a CUDA graph and replayed
 * by later calls with the same plans, buffers and parameters (new density
 * values in the same buffers are fine); the first use_graph call of a batch
 * runs without capture.  One batch per stream at a time.
 *
 * No counterpart in the reference, which builds one molecule per call
 * (electrolites/fastjk.py:276).
 */
typedef struct jk_batch jk_batch;
int jk_batch_create(int device, jk_batch **out);
int jk_batch_destroy(jk_batch *batch);
int jk_batch_build(jk_batch *batch, jk_plan *const *plans, int nplans,
                   const double *const *dms, const int *n_dm, int hermi,
                   int with_j, int with_k, double *const *vj, double *const *vk,
                   double mixed_threshold, int use_graph, void *stream);
/* Wait for the batch's work on stream; JK_ERR_RANGE names the plan index
 * whose density is beyond its plan's range. */
int jk_batch_sync(jk_batch *batch, void *stream);
/* As jk_last_counts, summed over the plans of the last batched build. */
int jk_batch_counts(jk_batch *batch, unsigned long long *quartets,
                    unsigned long long *prim_quartets,
                    unsigned long long *quartets_f32, int ncounts,
                    int *nclasses);
/* As jk_set_timing / jk_last_class_ms (no per-class times for graph
 * replays). */
int jk_batch_set_timing(jk_batch *batch, int enable);
int jk_batch_class_ms(jk_batch *batch, float *ms, int ncounts, int *launches);
/* As jk_plan_set_tuning, for the batch's builds. */
int jk_batch_set_tuning(jk_batch *batch, int cls, int tasks_per_sm,
                        int blocks_per_sm, int fp32);
/* Whether the last build replayed or captured a graph, and the batch's
 * device workspace. */
int jk_batch_stats(jk_batch *batch, int *graph_replayed, int *graph_captured,
                   long long *workspace_bytes);

const char *jk_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
