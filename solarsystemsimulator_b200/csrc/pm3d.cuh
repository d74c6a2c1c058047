// Shared pieces of the 3-D periodic particle mesh (pm3d.cu) and the learned
// correction (mlp.cu): the plan object, the CIC cell of a position, and the
// fused KDK epilogue both force passes end with.
#pragma once

#include "sss_internal.cuh"

#include <cufft.h>

struct sss_pm3 {
    sss_ctx* ctx;
    int n;              // mesh side
    double box;         // periodic box side
    float* rho;         // n^3 density (mass / h^3)
    float* lrho;        // n^3 log1p(rho / rho_mean): the correction network's inputs
    float2* rk;         // n * n * (n/2 + 1) spectrum of rho
    float2* ak;         // 3 spectra of the acceleration components (contiguous)
    float* acc;         // 3 n^3 acceleration meshes (contiguous)
    cufftHandle fwd;    // R2C n^3
    cufftHandle inv3;   // C2R n^3, batch 3
    double* tab;        // per-axis tables of the spectrum kernel: kd[n], k2[n], fac[n]
    int tab_deconv;     // parameters the tables were built for (-1: none yet)
    double tab_rs2;
};

// Particle state passed by value to kernels.
struct Pm3Parts {
    long long n;
    double* x[3];
    double* v[3];
    double* a[3];
    const double* m;
    double mass_const;
};

inline Pm3Parts pm3_parts(const sss_pm3_particles* s) {
    Pm3Parts p;
    p.n = s->n;
    for (int c = 0; c < 3; ++c) {
        p.x[c] = s->x[c];
        p.v[c] = s->v[c];
        p.a[c] = s->a[c];
    }
    p.m = s->m;
    p.mass_const = s->mass_const;
    return p;
}

struct Pm3Epi {
    int mode;           // SSS_PM3_FORCE / KICK / KICK_DRIFT
    double hdt, dt, box;
    float* snap;        // nullable: f32 row [x|y|z|vx|vy|vz]
};

// Lower CIC node (wrapped to [0, n)) and fractional offset along one axis:
// f = x n / box, i0 = floor(f), t = f - i0 (the deposit and the gather use
// this one stencil, so a particle never pulls on itself through the mesh
// weights; pm_kernel.py:63-90 clips instead, being isolated).
__device__ __forceinline__ void pm3_cell(double x, double inv_h, int n, int& i0, double& t) {
    const double f = x * inv_h;
    const double fl = floor(f);
    t = f - fl;
    int i = (int)fl;
    i %= n;
    if (i < 0) i += n;
    i0 = i;
}

__device__ __forceinline__ double pm3_wrap(double x, double box) { return x - box * floor(x / box); }

// The epilogue of a force pass for particle p with acceleration (ax, ay, az).
__device__ __forceinline__ void pm3_epilogue(const Pm3Parts& s, const Pm3Epi& e, long long p, double ax,
                                             double ay, double az) {
    s.a[0][p] = ax;
    s.a[1][p] = ay;
    s.a[2][p] = az;
    if (e.mode == SSS_PM3_FORCE) return;
    double v0 = s.v[0][p] + ax * e.hdt;
    double v1 = s.v[1][p] + ay * e.hdt;
    double v2 = s.v[2][p] + az * e.hdt;
    if (e.mode == SSS_PM3_KICK_DRIFT) {
        double x0 = s.x[0][p], x1 = s.x[1][p], x2 = s.x[2][p];
        if (e.snap) {
            const long long n = s.n;
            e.snap[p] = (float)x0;
            e.snap[n + p] = (float)x1;
            e.snap[2 * n + p] = (float)x2;
            e.snap[3 * n + p] = (float)v0;
            e.snap[4 * n + p] = (float)v1;
            e.snap[5 * n + p] = (float)v2;
        }
        v0 += ax * e.hdt;
        v1 += ay * e.hdt;
        v2 += az * e.hdt;
        s.x[0][p] = pm3_wrap(x0 + v0 * e.dt, e.box);
        s.x[1][p] = pm3_wrap(x1 + v1 * e.dt, e.box);
        s.x[2][p] = pm3_wrap(x2 + v2 * e.dt, e.box);
    } else if (e.snap) {
        const long long n = s.n;
        e.snap[p] = (float)s.x[0][p];
        e.snap[n + p] = (float)s.x[1][p];
        e.snap[2 * n + p] = (float)s.x[2][p];
        e.snap[3 * n + p] = (float)v0;
        e.snap[4 * n + p] = (float)v1;
        e.snap[5 * n + p] = (float)v2;
    }
    s.v[0][p] = v0;
    s.v[1][p] = v1;
    s.v[2][p] = v2;
}
