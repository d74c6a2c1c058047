// Pieces shared by the all-pairs translation units: the integrator epilogue
// every force kernel ends with (acceleration store, closing half kick,
// snapshot, next opening half kick and drift; reference
// backend/selfgrav_kernel.py:335-386) and the tensor-core force evaluation
// that allpairs.cu dispatches to (allpairs_tc.cu).
#pragma once

#include "sss_internal.cuh"

namespace sss_ap {

struct Epi {
    int mode;            // 0: write accelerations only; 1: integrator step
    int last;            // mode 1: no opening kick / drift after this force
    double4* acc;        // out: accelerations (both modes)
    double4* vel;        // mode 1
    double4* pos_nxt;    // mode 1: drifted positions
    float* snap;         // mode 1: snapshot row or nullptr
    double kc, ko, kd;   // closing kick, opening kick, drift factors
    int64_t n_src, n_tr; // snapshot layout
};

template <int D>
__device__ __forceinline__ void epilogue(const Epi& e, int64_t i, double ax, double ay,
                                         double az, const double4& p) {
    e.acc[i] = make_double4(ax, ay, az, 0.0);
    if (e.mode == 0) return;
    double4 v = e.vel[i];
    // closing half kick, as `vx[i] += a0 * (0.5 * dt)` (selfgrav_kernel.py:366-367)
    v.x += ax * e.kc;
    v.y += ay * e.kc;
    if (D == 3) v.z += az * e.kc;
    if (e.snap != nullptr) {
        if (i < e.n_src) {
            const int64_t n = e.n_src;
            e.snap[i] = (float)p.x;
            e.snap[n + i] = (float)p.y;
            if (D == 3) e.snap[2 * n + i] = (float)p.z;
            float* sv = e.snap + D * n;
            sv[i] = (float)v.x;
            sv[n + i] = (float)v.y;
            if (D == 3) sv[2 * n + i] = (float)v.z;
        } else {
            const int64_t t = i - e.n_src, m = e.n_tr;
            float* st = e.snap + 2 * D * e.n_src;
            st[t] = (float)p.x;
            st[m + t] = (float)p.y;
            if (D == 3) st[2 * m + t] = (float)p.z;
        }
    }
    double4 q = p;
    if (!e.last) {
        // next opening half kick + drift (selfgrav_kernel.py:335-346)
        v.x += ax * e.ko;
        v.y += ay * e.ko;
        if (D == 3) v.z += az * e.ko;
        q.x = p.x + v.x * e.kd;
        q.y = p.y + v.y * e.kd;
        if (D == 3) q.z = p.z + v.z * e.kd;
    }
    e.vel[i] = v;
    e.pos_nxt[i] = q;
}

// Force evaluation of SSS_PREC_MIXED_TC (allpairs_tc.cu): the pair terms as
// tensor-core products over tile-centred coordinates, f32 partial sums in
// tensor memory folded into f64. Same contract as the SIMT force_eval.
int force_eval_tc(sss_ctx* ctx, int dim, const double4* src, int64_t n_src, const double4* tgt, int64_t n_tgt,
                  double eps2, const Epi& epi, cudaStream_t stream);

}  // namespace sss_ap
