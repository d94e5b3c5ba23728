// markley.h — Markley quaternion mean: the dominant eigenvector of the
// symmetrised 4x4 moment matrix M = sum_i w_i q_i q_i^T (Markley, Cheng,
// Crassidis, Oshman, "Averaging quaternions", JGCD 2007), in FP64, for host
// and device.
//
// Semantics follow crates/pf_core/src/types.rs:128-143: symmetrise
// (M^T + M)/2, take the eigenvector of the largest eigenvalue (first index on
// ties), normalise, flip to w >= 0.  The dominant eigenvector comes from
// repeated squaring of M (a few hundred FP64 operations with no divisions in
// the loop, so a single GPU thread finishes it in about a microsecond),
// checked by its Rayleigh residual; near-degenerate spectra fall back to the
// cyclic Jacobi method (Golub & Van Loan, "Matrix Computations", section
// 8.5).  nalgebra's tridiagonal QR returns the same unit eigenvector up to
// sign for a simple top eigenvalue, and the sign is canonicalised.
#pragma once

#ifdef __CUDACC__
#define PFB_HD __host__ __device__
#else
#define PFB_HD
#endif

#include <math.h>

namespace pfb {

// Eigen-decomposition of a symmetric 4x4 matrix a (row-major, destroyed).
// On return a holds the eigenvalues on its diagonal and v the eigenvectors
// as columns.  Returns the number of sweeps used.
PFB_HD inline int jacobi_eig4(double a[16], double v[16]) {
    for (int i = 0; i < 16; ++i) v[i] = (i % 5 == 0) ? 1.0 : 0.0;
    int sweep = 0;
    for (; sweep < 64; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int p = 0; p < 4; ++p) {
            diag += a[p * 4 + p] * a[p * 4 + p];
            for (int q = p + 1; q < 4; ++q) off += a[p * 4 + q] * a[p * 4 + q];
        }
        if (!(off > 1e-32 * diag) || off == 0.0) break;
        for (int p = 0; p < 3; ++p) {
            for (int q = p + 1; q < 4; ++q) {
                const double apq = a[p * 4 + q];
                if (apq == 0.0) continue;
                const double app = a[p * 4 + p], aqq = a[q * 4 + q];
                // Rutishauser's stable rotation: t = tan(phi) of the smaller
                // root of t^2 + 2 theta t - 1 = 0.
                const double theta = (aqq - app) / (2.0 * apq);
                const double t =
                    (theta >= 0.0 ? 1.0 : -1.0) /
                    (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0);
                const double s = t * c;
                for (int k = 0; k < 4; ++k) {
                    const double akp = a[k * 4 + p], akq = a[k * 4 + q];
                    a[k * 4 + p] = c * akp - s * akq;
                    a[k * 4 + q] = s * akp + c * akq;
                }
                for (int k = 0; k < 4; ++k) {
                    const double apk = a[p * 4 + k], aqk = a[q * 4 + k];
                    a[p * 4 + k] = c * apk - s * aqk;
                    a[q * 4 + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 4; ++k) {
                    const double vkp = v[k * 4 + p], vkq = v[k * 4 + q];
                    v[k * 4 + p] = c * vkp - s * vkq;
                    v[k * 4 + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    return sweep;
}

// Dominant eigenvector of a symmetric positive semi-definite 4x4 matrix by
// repeated squaring (the power method on M^(2^k)): after 12 squarings the
// other eigen-directions are damped by (lambda2/lambda1)^4096.  The squaring
// stops earlier once the trace-normalised matrix P is rank one to rounding,
// 1 - tr(P^2) < 1e-14 (tr(P^2) is the sum of the squared normalised
// eigenvalues; it is 1 - 2e for a remainder e off the top direction), which
// for a particle cloud takes three or four squarings.  Accepted only
// when the Rayleigh residual |M v - (v'Mv) v| is below 1e-13 |M|; returns
// false otherwise (near-degenerate top eigenvalue), and the caller falls back
// to the Jacobi solve.
PFB_HD inline bool dominant_eigvec_psd4(const double a[16], double v[4]) {
    double p[16], t[16];
    double tr = a[0] + a[5] + a[10] + a[15];
    if (!(tr > 0.0)) return false;
    const double itr = 1.0 / tr;
    for (int i = 0; i < 16; ++i) p[i] = a[i] * itr;
    for (int s = 0; s < 12; ++s) {
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c)
                t[r * 4 + c] = p[r * 4 + 0] * p[0 * 4 + c] + p[r * 4 + 1] * p[1 * 4 + c] +
                               p[r * 4 + 2] * p[2 * 4 + c] + p[r * 4 + 3] * p[3 * 4 + c];
        const double tt = t[0] + t[5] + t[10] + t[15];
        if (!(tt > 0.0)) return false;
        const double itt = 1.0 / tt;
        for (int i = 0; i < 16; ++i) p[i] = t[i] * itt;
        if (tt > 1.0 - 1e-14) break;
    }
    // p ~ v v^T: take the column with the largest diagonal entry.
    int c = 0;
    for (int i = 1; i < 4; ++i)
        if (p[i * 4 + i] > p[c * 4 + c]) c = i;
    double x[4] = {p[0 * 4 + c], p[1 * 4 + c], p[2 * 4 + c], p[3 * 4 + c]};
    // two power steps with the original matrix polish the direction
    for (int it = 0; it < 2; ++it) {
        double y[4];
        for (int r = 0; r < 4; ++r)
            y[r] = a[r * 4 + 0] * x[0] + a[r * 4 + 1] * x[1] + a[r * 4 + 2] * x[2] +
                   a[r * 4 + 3] * x[3];
        const double ny = sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2] + y[3] * y[3]);
        if (!(ny > 0.0)) return false;
        for (int r = 0; r < 4; ++r) x[r] = y[r] / ny;
    }
    double y[4];
    for (int r = 0; r < 4; ++r)
        y[r] = a[r * 4 + 0] * x[0] + a[r * 4 + 1] * x[1] + a[r * 4 + 2] * x[2] +
               a[r * 4 + 3] * x[3];
    const double lam = x[0] * y[0] + x[1] * y[1] + x[2] * y[2] + x[3] * y[3];
    double res = 0.0;
    for (int r = 0; r < 4; ++r) res += (y[r] - lam * x[r]) * (y[r] - lam * x[r]);
    if (!(sqrt(res) <= 1e-13 * tr)) return false;
    for (int r = 0; r < 4; ++r) v[r] = x[r];
    return true;
}

// Mean quaternion (w,x,y,z) from the 10 packed upper-triangle moments
// M00,M01,M02,M03,M11,M12,M13,M22,M23,M33 (the layout of pfc_est_sums
// out[3..12], unpacked by crates/pf_core/src/cuda.rs:277-285).
PFB_HD inline void markley_mean(const double m10[10], double q_out[4]) {
    double a[16], v[16];
    int e = 0;
    for (int r = 0; r < 4; ++r)
        for (int c = r; c < 4; ++c) {
            a[r * 4 + c] = m10[e];
            a[c * 4 + r] = m10[e];
            ++e;
        }
    double q[4];
    if (!dominant_eigvec_psd4(a, q)) {
        jacobi_eig4(a, v);
        int idx = 0;
        for (int i = 1; i < 4; ++i)
            if (a[i * 4 + i] > a[idx * 4 + idx]) idx = i;
        for (int r = 0; r < 4; ++r) q[r] = v[r * 4 + idx];
    }
    double nrm = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    if (!(nrm > 0.0)) {
        q_out[0] = 1.0;
        q_out[1] = q_out[2] = q_out[3] = 0.0;
        return;
    }
    double sgn = (q[0] < 0.0) ? -1.0 : 1.0;
    for (int i = 0; i < 4; ++i) q_out[i] = sgn * q[i] / nrm;
}

#ifdef __CUDACC__
// The serial solve as a call of its own (the rare fallback below), so its
// registers do not count against its caller.
static __device__ __noinline__ void markley_mean_serial(const double* m10, double* q_out) {
    markley_mean(m10, q_out);
}

// markley_mean by one warp: lanes 4r + c (r, c < 4) of the first 16 hold
// element (r, c) of the 4x4 matrix, so a squaring is four shuffled products
// per lane instead of 64 serial ones; the same method and acceptance test as
// dominant_eigvec_psd4, and the same serial Jacobi fallback (one lane) for a
// near-degenerate top eigenvalue.  Every lane of the warp must call it; the
// result is valid in every lane.
__device__ inline void markley_mean_warp(const double m10[10], double q_out[4]) {
    const unsigned full = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const int r = (lane >> 2) & 3, c = lane & 3;
    const int lo = r < c ? r : c, hi = r < c ? c : r;
    const double a = m10[lo * 4 - lo * (lo - 1) / 2 + (hi - lo)];  // a[r][c]
    auto at = [&](double v, int rr, int cc) { return __shfl_sync(full, v, rr * 4 + cc); };
    auto trace = [&](double v) {
        return at(v, 0, 0) + at(v, 1, 1) + at(v, 2, 2) + at(v, 3, 3);
    };
    const double tr = trace(a);
    bool ok = tr > 0.0;
    double x[4] = {0.0, 0.0, 0.0, 0.0};
    if (ok) {
        const double itr = 1.0 / tr;
        double pm = a * itr;
        for (int s = 0; s < 12 && ok; ++s) {
            const double t = at(pm, r, 0) * at(pm, 0, c) + at(pm, r, 1) * at(pm, 1, c) +
                             at(pm, r, 2) * at(pm, 2, c) + at(pm, r, 3) * at(pm, 3, c);
            const double tt = trace(t);
            ok = tt > 0.0;
            pm = t * (1.0 / tt);
            if (tt > 1.0 - 1e-14) break;  // warp-uniform: every lane has tt
        }
        if (ok) {
            // the column of the largest diagonal entry, then two power steps
            // with the original matrix
            int cb = 0;
            double db = at(pm, 0, 0);
            for (int i = 1; i < 4; ++i) {
                const double d = at(pm, i, i);
                if (d > db) {
                    db = d;
                    cb = i;
                }
            }
            for (int i = 0; i < 4; ++i) x[i] = at(pm, i, cb);
            for (int it = 0; it < 2 && ok; ++it) {
                double y[4];
                for (int i = 0; i < 4; ++i)
                    y[i] = at(a, i, 0) * x[0] + at(a, i, 1) * x[1] + at(a, i, 2) * x[2] +
                           at(a, i, 3) * x[3];
                const double ny = sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2] + y[3] * y[3]);
                ok = ny > 0.0;
                for (int i = 0; i < 4; ++i) x[i] = y[i] / ny;
            }
            if (ok) {
                double y[4];
                for (int i = 0; i < 4; ++i)
                    y[i] = at(a, i, 0) * x[0] + at(a, i, 1) * x[1] + at(a, i, 2) * x[2] +
                           at(a, i, 3) * x[3];
                const double lam = x[0] * y[0] + x[1] * y[1] + x[2] * y[2] + x[3] * y[3];
                double res = 0.0;
                for (int i = 0; i < 4; ++i) res += (y[i] - lam * x[i]) * (y[i] - lam * x[i]);
                ok = sqrt(res) <= 1e-13 * tr;
            }
        }
    }
    if (!ok) {
        // near-degenerate spectrum: the serial solve, by lane 0
        double q[4];
        if (lane == 0) markley_mean_serial(m10, q);
        for (int i = 0; i < 4; ++i) q_out[i] = __shfl_sync(full, q[i], 0);
        return;
    }
    const double nrm = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + x[3] * x[3]);
    if (!(nrm > 0.0)) {
        q_out[0] = 1.0;
        q_out[1] = q_out[2] = q_out[3] = 0.0;
        return;
    }
    const double sgn = (x[0] < 0.0) ? -1.0 : 1.0;
    for (int i = 0; i < 4; ++i) q_out[i] = sgn * x[i] / nrm;
}

// markley_mean_warp as a call of its own: not inlined, so its registers do
// not count against the streaming loop of the kernel that calls it at its
// end.  Every lane of the calling warp must call it.
static __device__ __noinline__ void markley_mean_warp_call(const double* m10, double* q_out) {
    markley_mean_warp(m10, q_out);
}
#endif

}  // namespace pfb
