// Host-side launch interface between the plan/build driver (jk_api.cu) and
// the generated per-class translation units.
#pragma once
#include <cuda_runtime.h>
#include "jk_device.cuh"

#define JK_MAX_DEVICES 64

struct LaunchCfg {
    cudaStream_t stream;
    int device;            // current device ordinal (< JK_MAX_DEVICES)
    int num_sms;
    int blocks_per_sm;     // cap on resident blocks per SM (0: occupancy limit)
    int configure_only;    // 1: set the kernel's attributes, launch nothing
    char *msg;             // 256 bytes: launch failure details
};

// a: the launch's part of the class; views: host copies of its a.nvl views
typedef int (*ClassLauncher)(const ClassArgs &a, const PlanView *views, const LaunchCfg &cfg);

struct ClassEntry {
    int bra_class, ket_class;     // pair-class indices la*(la+1)/2 + lb
    int li, lj, lk, ll;
    int form;                     // 0 register form, 1 team form
    int team_threads;
    int fp32_default;             // mixed builds run FP32 quartets here by default
    int md;                       // a McMurchie-Davidson J kernel exists (J-only builds)
    int md_default;               // J-only builds take it by default
    ClassLauncher launch;
};

// J engine, per pair class: the x-space densities D~_P = H^P^T (D+D^T)_P of
// every pair of the class, and the transfer of their x-space J back into the
// half-J accumulators, J_h(P) += H^P J~_P (one thread per pair and density).
struct PairArgs {
    const PairRec *pairs;         // the class's pairs
    int npairs;
    int n_j, nao;
    const double *ds;             // D + D^T, n_j x nao x nao
    double *Jh;                   // half-J accumulators, n_j x nao x nao
    double *dt;                   // x-space densities
    const double *jx;             // x-space J
};
typedef int (*PairLauncher)(const PairArgs &a, cudaStream_t st);

struct PairEntry {
    int pair_class, la, lb, nx;
    PairLauncher dens, post;
};
