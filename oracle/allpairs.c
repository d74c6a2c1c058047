/*
 * CPU oracle — TEST INFRASTRUCTURE ONLY (never linked into libsss or the
 * product path). Plain-C restatement of the reference's all-pairs Plummer
 * force, used by tests/ and by bench.py's CPU baseline.
 *
 * Follows `beschleunigung` (reference backend/selfgrav_kernel.py:222-260):
 * each target sums its sources in ascending index order,
 *   r2  = dx*dx + dy*dy (+ dz*dz) + eps2
 *   inv = 1/sqrt(r2)              (the reference's rsqrt, :252)
 *   f   = (G m) * inv * inv * inv (:253, G m premultiplied in the record)
 *   a  += f * d                   (:254-255)
 * with no FMA contraction (-ffp-contract=off), so results are the IEEE
 * evaluation of that expression order. The self term contributes 0 (d = 0).
 * Records are {x, y, z, Gm} doubles; dim = 2 ignores z.
 *
 * Also: the Plummer potential (test_selfgrav.py:54-63) and the hot-loop
 * free functions used by the parity tests. Parallel over targets with
 * OpenMP; the per-target order is independent of the thread count.
 */
#include <math.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

void oracle_allpairs_accel(int dim, const double* src4, int64_t n_src,
                           const double* tgt4, int64_t n_tgt, double* acc4,
                           double eps2, int nthreads) {
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 64)
    for (int64_t i = 0; i < n_tgt; ++i) {
        const double px = tgt4[4 * i], py = tgt4[4 * i + 1], pz = tgt4[4 * i + 2];
        double ax = 0.0, ay = 0.0, az = 0.0;
        for (int64_t j = 0; j < n_src; ++j) {
            const double* s = src4 + 4 * j;
            const double dx = s[0] - px;
            const double dy = s[1] - py;
            double r2;
            double dz = 0.0;
            if (dim == 3) {
                dz = s[2] - pz;
                r2 = dx * dx + dy * dy + dz * dz + eps2;
            } else {
                r2 = dx * dx + dy * dy + eps2;
            }
            const double inv = 1.0 / sqrt(r2);
            const double f = s[3] * inv * inv * inv;
            ax += f * dx;
            ay += f * dy;
            if (dim == 3) az += f * dz;
        }
        acc4[4 * i] = ax;
        acc4[4 * i + 1] = ay;
        acc4[4 * i + 2] = az;
        acc4[4 * i + 3] = 0.0;
    }
}

/* Sum of |term| per component (cancellation-aware error scale). */
void oracle_allpairs_absterm(int dim, const double* src4, int64_t n_src,
                             const double* tgt4, int64_t n_tgt, double* abs4,
                             double eps2, int nthreads) {
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 64)
    for (int64_t i = 0; i < n_tgt; ++i) {
        const double px = tgt4[4 * i], py = tgt4[4 * i + 1], pz = tgt4[4 * i + 2];
        double ax = 0.0, ay = 0.0, az = 0.0;
        for (int64_t j = 0; j < n_src; ++j) {
            const double* s = src4 + 4 * j;
            const double dx = s[0] - px, dy = s[1] - py;
            const double dz = (dim == 3) ? s[2] - pz : 0.0;
            const double r2 = dx * dx + dy * dy + dz * dz + eps2;
            const double inv = 1.0 / sqrt(r2);
            const double f = fabs(s[3]) * inv * inv * inv;
            ax += f * fabs(dx);
            ay += f * fabs(dy);
            az += f * fabs(dz);
        }
        abs4[4 * i] = ax;
        abs4[4 * i + 1] = ay;
        abs4[4 * i + 2] = az;
        abs4[4 * i + 3] = 0.0;
    }
}

/* phi_t = -sum_s Gm_s / sqrt(|d|^2 + eps2), self term included. */
void oracle_allpairs_potential(int dim, const double* src4, int64_t n_src,
                               const double* tgt4, int64_t n_tgt, double* phi,
                               double eps2, int nthreads) {
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 64)
    for (int64_t i = 0; i < n_tgt; ++i) {
        const double px = tgt4[4 * i], py = tgt4[4 * i + 1], pz = tgt4[4 * i + 2];
        double acc = 0.0;
        for (int64_t j = 0; j < n_src; ++j) {
            const double* s = src4 + 4 * j;
            const double dx = s[0] - px, dy = s[1] - py;
            const double dz = (dim == 3) ? s[2] - pz : 0.0;
            const double r2 = dx * dx + dy * dy + dz * dz + eps2;
            acc += s[3] / sqrt(r2);
        }
        phi[i] = -acc;
    }
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
