// brdc_secular.cuh -- one secular root as a resumable state machine.
//
// Solves  f(lambda) = 1/rho + sum_j z_j^2 / (d_j - lambda) = 0  for root i of
// a deflated rank-one update (poles d_0 < ... < d_{K-1}, rho > 0): root
// i < K-1 lies in (d_i, d_{i+1}), root K-1 in (d_{K-1}, d_{K-1}+rho*|z|^2].
//
// The iteration is Ren-Cang Li's "middle way" / "fixed weight" rational
// scheme with bisection safeguards (R.-C. Li, "Solving secular equations
// stably and efficiently", LAPACK Working Note 89, 1994), the scheme LAPACK
// DLAED4 implements and the reference calls for every root
// (cpu/src/dlaed4_br.f:59; its GPU prototype restates it without the
// three-pole step in gpu/src/tridiag_solver_secular.cuh:404-601,953-1085).
// This file is written for a GPU that evaluates the O(K) sums of many roots
// in one sweep over shared-memory tiles of poles:
//   * the state is advanced between sweeps (sec_after_sweep), so a thread
//     block can interleave the sweeps of all its roots;
//   * every delta is recomputed from the compact pair (origin, tau),
//     delta_j = (d_j - d_org) - tau, instead of being updated in place, so no
//     O(K) delta column is stored per root (the compact ORG/TAU
//     representation of cpu/src/dlaed4_br.f:15-26,95-103);
//   * the sweep excludes the two bracketing poles p, p+1; the root adds
//     their terms itself so they are never cancelled against the rest.
// The error bound is LAPACK's running-sum bound for the summation order the
// sweep actually uses.
#pragma once

#include <cmath>

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#endif

namespace brdc {

// Default cap on the iterations of one root; a handle may set another
// (brdc_set_limits), which the kernels read from the workspace header.
constexpr int kSecularMaxIter = 64;

// 1/x for the pole-root pair loops.  IEEE division carries a branch to its
// special-case path, which keeps the compiler from overlapping the
// divisions of consecutive poles; this form has none.  It starts from the
// hardware estimate rcp.approx.ftz.f64 and takes one third-order step,
// r <- r + r (e + e^2) with e = 1 - x r (the series 1/x = r / (1 - e) cut
// after e^2), which cubes the estimate's relative error; the result is
// within 1 ulp of 1/x and almost always the correctly rounded value
// (tests/test_rcp_gpu.py measures it against IEEE division).  On B200 this
// takes three fused multiply-adds where two Newton-Raphson steps took four:
// 31% more reciprocals per second in a throughput probe, Toeplitz 65,536
// 23.7 -> 22.2 ms.  x must be a normal, finite, nonzero
// double whose reciprocal is normal: every delta of these loops is a
// difference of distinct poles and roots of order ||T||.  Host builds
// divide.
__host__ __device__ inline double brdc_rcp(double x) {
#ifdef __CUDA_ARCH__
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    const double e = fma(-x, r, 1.0);
    return fma(r, fma(e, e, e), r);
#else
    return 1.0 / x;
#endif
}

// Two factors of a Loewner product, (d_i - lambda_j) / (d_i - d_j) for two
// poles j, with one reciprocal of the product of their denominators.  The
// denominators are distinct poles' differences (or 1 for j = i), of order
// ||T|| down to the deflation tolerance, and the numerators of order ||T||
// down to a root's distance from its pole, so neither product comes near
// the ends of the double range.  The reciprocal is the pair loops' dearest
// operation (a quarter-rate estimate and three FMAs), and one per two
// factors takes about a third off the product's cost.
__host__ __device__ inline double lowner_pair(double num1, double den1, double num2,
                                              double den2) {
    return (num1 * num2) * brdc_rcp(den1 * den2);
}

// The secular vector entries u = w / delta of two poles, with one
// reciprocal of the product of their deltas.  The deltas are distances of
// one root from distinct poles, so at most one of them is tiny and the
// product stays inside the double range.  A zero delta (a root on a pole,
// reachable only through underflow) gives u = 0, as the single form does.
__host__ __device__ inline void row_pair(double w1, double dl1, double w2, double dl2,
                                         double *u1, double *u2) {
    const double e1 = dl1 != 0.0 ? dl1 : 1.0, e2 = dl2 != 0.0 ? dl2 : 1.0;
    const double inv = brdc_rcp(e1 * e2);
    *u1 = dl1 != 0.0 ? w1 * (e2 * inv) : 0.0;
    *u2 = dl2 != 0.0 ? w2 * (e1 * inv) : 0.0;
}

struct SecSums {
    double psi;   // sum_{j < p} z_j^2 / delta_j
    double dpsi;  // sum_{j < p} z_j^2 / delta_j^2
    double phi;   // sum_{j > p+1} z_j^2 / delta_j
    double dphi;  // sum_{j > p+1} z_j^2 / delta_j^2
    double err;   // running-sum rounding bound of the two partial sums
};

__host__ __device__ inline void sec_zero(SecSums &s) {
    s.psi = 0.0;
    s.dpsi = 0.0;
    s.phi = 0.0;
    s.dphi = 0.0;
    s.err = 0.0;
}

struct SecRoot {
    // problem (fixed)
    int i;         // root index
    int p;         // left model pole (i, or K-2 for the last root)
    int last;      // 1 for the root right of the last pole
    double dp, dq; // d_p, d_{p+1}
    double zp2, zq2;
    double rhoinv;
    double hi0;    // last root: rho * |z|^2 (upper bound of tau)
    // iteration state
    int stage;     // 0: midpoint sums pending, 1: iterating, 2: done
    int org;       // origin pole index (p or p+1)
    double dorg;   // d_org
    double tau;    // lambda = d_org + tau
    double lo, hi; // bracket of tau
    double prevw;
    int iter;
    int swtch;     // 1: middle way, 0: fixed weight
    int failed;
    // evaluation point of the next sweep: delta_j = (d_j - eorg_d) - etau
    double eorg_d;
    double etau;
};

// Set up root i (0-based) of a problem with K >= 2 poles.  d and z are the
// pole and weight arrays (only d_p, d_{p+1}, z_p, z_{p+1} are read).
// The fields of root i that never change (a solver that parks the iteration
// state between sweeps rebuilds them from the problem instead of storing).
// rhoinv = 1 / rho, which a caller that rebuilds the fields every sweep
// computes once per node.
__host__ __device__ inline void sec_init_static(SecRoot &r, int i, int K, const double *d,
                                                const double *z, double rho, double rhoinv,
                                                double znorm2) {
    r.i = i;
    r.last = (i == K - 1) ? 1 : 0;
    r.p = r.last ? K - 2 : i;
    r.dp = d[r.p];
    r.dq = d[r.p + 1];
    r.zp2 = z[r.p] * z[r.p];
    r.zq2 = z[r.p + 1] * z[r.p + 1];
    r.rhoinv = rhoinv;
    r.hi0 = rho * znorm2;
}

__host__ __device__ inline void sec_init_static(SecRoot &r, int i, int K, const double *d,
                                                const double *z, double rho, double znorm2) {
    sec_init_static(r, i, K, d, z, rho, 1.0 / rho, znorm2);
}

// The fields that a sweep and sec_after_sweep advance.
struct SecDyn {
    double dorg, tau, lo, hi, prevw, eorg_d, etau;
    int stage, org, iter, swtch, failed;
};

__host__ __device__ inline void sec_park(const SecRoot &r, SecDyn &q) {
    q.dorg = r.dorg;
    q.tau = r.tau;
    q.lo = r.lo;
    q.hi = r.hi;
    q.prevw = r.prevw;
    q.eorg_d = r.eorg_d;
    q.etau = r.etau;
    q.stage = r.stage;
    q.org = r.org;
    q.iter = r.iter;
    q.swtch = r.swtch;
    q.failed = r.failed;
}

__host__ __device__ inline void sec_unpark(SecRoot &r, const SecDyn &q) {
    r.dorg = q.dorg;
    r.tau = q.tau;
    r.lo = q.lo;
    r.hi = q.hi;
    r.prevw = q.prevw;
    r.eorg_d = q.eorg_d;
    r.etau = q.etau;
    r.stage = q.stage;
    r.org = q.org;
    r.iter = q.iter;
    r.swtch = q.swtch;
    r.failed = q.failed;
}

__host__ __device__ inline void sec_init(SecRoot &r, int i, int K,
                                         const double *d, const double *z,
                                         double rho, double znorm2) {
    sec_init_static(r, i, K, d, z, rho, znorm2);
    r.stage = 0;
    r.iter = 0;
    r.swtch = 0;
    r.failed = 0;
    r.prevw = 0.0;
    if (r.last) {
        r.org = r.p + 1;
        r.dorg = r.dq;
        r.lo = 0.0;
        r.hi = r.hi0;
        r.eorg_d = r.dq;
        r.etau = 0.5 * r.hi0;
    } else {
        r.org = r.p;
        r.dorg = r.dp;
        const double mid = 0.5 * (r.dq - r.dp);
        r.lo = 0.0;
        r.hi = mid;
        r.eorg_d = r.dp;
        r.etau = mid;
    }
    r.tau = r.etau;
}

// One term of the sweep for pole j (d_j, z_j).  Poles p and p+1 are skipped.
// Branch-free, because the lanes of a warp serve roots with different p.
__host__ __device__ inline void sec_accum(SecSums &s, const SecRoot &r, int j,
                                          double dj, double zj) {
    const bool skip = (j == r.p) || (j == r.p + 1);
    const bool left = j < r.p;
    const double delta = (dj - r.eorg_d) - r.etau;
    double t = zj * brdc_rcp(skip ? 1.0 : delta);
    t = skip ? 0.0 : t;
    const double term = zj * t;
    const double t2 = t * t;
    s.psi += left ? term : 0.0;
    s.dpsi += left ? t2 : 0.0;
    s.phi += left ? 0.0 : term;
    s.dphi += left ? 0.0 : t2;
    s.err += skip ? 0.0 : (left ? -s.psi : s.phi);
}

// The same term for a pole known to lie left of p (j < p) or right of p+1
// (j > p+1): callers use these for tiles wholly on one side of every root
// they serve, which removes the per-element selects of sec_accum.  The
// arithmetic is identical to sec_accum's for such poles.
__host__ __device__ inline void sec_accum_left(SecSums &s, const SecRoot &r,
                                               double dj, double zj) {
    const double delta = (dj - r.eorg_d) - r.etau;
    const double t = zj * brdc_rcp(delta);
    s.psi += zj * t;
    s.dpsi += t * t;
    s.err -= s.psi;
}

__host__ __device__ inline void sec_accum_right(SecSums &s, const SecRoot &r,
                                                double dj, double zj) {
    const double delta = (dj - r.eorg_d) - r.etau;
    const double t = zj * brdc_rcp(delta);
    s.phi += zj * t;
    s.dphi += t * t;
    s.err += s.phi;
}

// Combine partial sums of two lanes (the tree adds its own rounding).  Every
// operation is commutative in (a, b), so the lanes of a butterfly reduction
// end with bit-identical sums and take identical branches afterwards.
__host__ __device__ inline void sec_combine(SecSums &a, const SecSums &b) {
    a.psi = a.psi + b.psi;
    a.dpsi = a.dpsi + b.dpsi;
    a.phi = a.phi + b.phi;
    a.dphi = a.dphi + b.dphi;
    a.err = (a.err + b.err) + (fabs(a.psi) + a.phi);
}

__host__ __device__ inline double sec_clamp_tau(double t, double lo, double hi) {
    if (!(t > lo && t < hi)) {
        t = 0.5 * (lo + hi);
    }
    return t;
}

// Advance the state after a sweep evaluated at (eorg_d, etau).  Returns the
// new stage (2 once converged or failed).  A root still unconverged after
// max_iter iterations, or whose secular function evaluates to NaN, is
// finished with r.failed set.
__host__ __device__ inline int sec_after_sweep(SecRoot &r, const SecSums &s,
                                               double eps, int max_iter = kSecularMaxIter) {
    if (r.stage == 2) {
        return 2;
    }
    if (r.stage == 0) {
        // Initial guess from the two bracketing poles with the rest of the
        // sum frozen at the evaluation point.
        const double c = r.rhoinv + s.psi + s.phi;
        if (!r.last) {
            const double del = r.dq - r.dp;
            const double mid = r.etau;
            const double w = c + r.zp2 / (-mid) + r.zq2 / ((r.dq - r.dp) - mid);
            double tau;
            if (w > 0.0) {
                // root in (d_p, mid): origin p
                r.org = r.p;
                r.dorg = r.dp;
                r.lo = 0.0;
                r.hi = mid;
                const double a = c * del + r.zp2 + r.zq2;
                const double b = r.zp2 * del;
                const double disc = sqrt(fabs(a * a - 4.0 * b * c));
                tau = (a > 0.0) ? 2.0 * b / (a + disc) : (a - disc) / (2.0 * c);
            } else {
                // root in [mid, d_q): origin p+1
                r.org = r.p + 1;
                r.dorg = r.dq;
                r.lo = -mid;
                r.hi = 0.0;
                const double a = c * del - r.zp2 - r.zq2;
                const double b = r.zq2 * del;
                const double disc = sqrt(fabs(a * a + 4.0 * b * c));
                tau = (a < 0.0) ? 2.0 * b / (a - disc) : -(a + disc) / (2.0 * c);
            }
            tau = sec_clamp_tau(tau, r.lo, r.hi);
            // Two safeguarded Newton steps on the model that also keeps the
            // slope of the rest of the sum at the midpoint,
            //   f(t) = c + B (t - t_mid) + zp2 / (e_p - t) + zq2 / (e_q - t),
            // B = dpsi + dphi.  When both bracketing weights are tiny the
            // two-pole guess sits on a pole while the root lies where the
            // rest of the sum crosses zero; the slope moves it there (host
            // measurements on merges of random tridiagonals: 3.44 -> 3.31
            // sweeps per root, the slowest roots 12 -> 9-10).  f increases
            // on the bracket, so the steps keep to it.
            {
                const bool orgati = (r.org == r.p);
                const double ep = orgati ? 0.0 : -del, eq = orgati ? del : 0.0;
                const double tm = orgati ? mid : -mid;
                const double B = s.dpsi + s.dphi;
                double lo = r.lo, hi = r.hi;
                // A second start: the zero of the rest of the sum alone,
                // t_mid - c / B.  Where both bracketing weights are tiny the
                // root sits there, and Newton steps from the two-pole guess
                // on a pole only double their distance to it per step.  The
                // start whose model value is nearer zero is kept (host
                // measurements on merges of random tridiagonals of 64 and
                // 256 rows: roots taking 7 or more sweeps 3.9% -> 1.7%).
                {
                    const double tl = tm - c * brdc_rcp(B);
                    if (tl > lo && tl < hi) {
                        const double fl = c + B * (tl - tm) + r.zp2 * brdc_rcp(ep - tl) +
                                          r.zq2 * brdc_rcp(eq - tl);
                        const double fg = c + B * (tau - tm) + r.zp2 * brdc_rcp(ep - tau) +
                                          r.zq2 * brdc_rcp(eq - tau);
                        if (fabs(fl) < fabs(fg)) {
                            tau = tl;
                        }
                    }
                }
#pragma unroll
                for (int it = 0; it < 2; ++it) {
                    // tau lies strictly inside the bracket, so both
                    // distances to the poles are nonzero
                    const double r1 = brdc_rcp(ep - tau), r2 = brdc_rcp(eq - tau);
                    const double t1 = r.zp2 * r1, t2 = r.zq2 * r2;
                    const double f = c + B * (tau - tm) + t1 + t2;
                    const double fp = B + t1 * r1 + t2 * r2;
                    if (f > 0.0) {
                        hi = tau;
                    } else {
                        lo = tau;
                    }
                    double tn = tau - f * brdc_rcp(fp);
                    if (!(tn > lo && tn < hi)) {
                        tn = 0.5 * (lo + hi);
                    }
                    tau = tn;
                }
            }
            r.tau = tau;
        } else {
            const double del = r.dq - r.dp;
            const double mid = r.etau;
            const double w = c + r.zp2 / ((r.dp - r.dq) - mid) + r.zq2 / (-mid);
            if (w <= 0.0) {
                r.lo = mid;
                r.hi = r.hi0;
            } else {
                r.lo = 0.0;
                r.hi = mid;
            }
            double tau = 0.5 * (r.lo + r.hi);
            if (c > 0.0) {
                const double a = c * del - r.zp2 - r.zq2;
                const double b = r.zq2 * del;
                const double disc = sqrt(fabs(a * a + 4.0 * b * c));
                const double t2 = (a <= 0.0) ? (disc - a) / (2.0 * c)
                                             : 2.0 * b / (a + disc);
                if (t2 > r.lo && t2 <= r.hi) {
                    tau = t2;
                } else if (!(t2 > r.lo)) {
                    tau = 0.5 * (r.lo + r.hi);
                } else {
                    tau = r.hi;
                }
            }
            r.tau = tau;
        }
        r.stage = 1;
        r.iter = 0;
        r.eorg_d = r.dorg;
        r.etau = r.tau;
        return 1;
    }

    // stage 1: sums at (dorg, tau).  This update is the serial part of every
    // iteration, so its quotients are reciprocals (brdc_rcp, no special-case
    // branch) times the numerator: deltas are nonzero (tau stays strictly
    // inside its bracket), and the model denominators are nonzero on the
    // branches that take them.
    r.iter += 1;
    const double tau = r.tau;
    const double dlp = (r.dp - r.dorg) - tau; // delta_p
    const double dlq = (r.dq - r.dorg) - tau; // delta_{p+1}
    const double rp = brdc_rcp(dlp);
    const double rq = brdc_rcp(dlq);
    const double tp = r.zp2 * rp;  // z_p^2 / delta_p
    const double tq = r.zq2 * rq;
    const double dtp = tp * rp;    // z_p^2 / delta_p^2
    const double dtq = tq * rq;
    const double psi_f = s.psi + tp;
    const double phi_f = s.phi + tq;
    const double dpsi_f = s.dpsi + dtp;
    const double dphi_f = s.dphi + dtq;
    const double w = r.rhoinv + psi_f + phi_f;
    const double dw = dpsi_f + dphi_f;

    double erretm;
    if (!r.last) {
        double psil = s.psi, phil = s.phi, err = s.err, torg;
        if (r.org == r.p) {
            phil += tq;
            err += phil;
            torg = tp;
        } else {
            psil += tp;
            err += fabs(psil);
            torg = tq;
        }
        erretm = 8.0 * (phil - psil) + err + 2.0 * r.rhoinv +
                 3.0 * fabs(torg) + fabs(tau) * dw;
    } else {
        const double psil = s.psi + tp;
        const double err = s.err + fabs(psil);
        erretm = 8.0 * (-tq - psil) + err - tq + r.rhoinv + fabs(tau) * dw;
    }

    if (!(w == w)) {
        // NaN: tau on a pole (a zero delta) or non-finite data; no step can
        // follow from it
        r.failed = 1;
        r.stage = 2;
        return 2;
    }
    if (fabs(w) <= eps * erretm) {
        r.stage = 2;
        return 2;
    }
    if (w <= 0.0) {
        r.lo = (tau > r.lo) ? tau : r.lo;
    } else {
        r.hi = (tau < r.hi) ? tau : r.hi;
    }
    if (r.hi - r.lo <= 2.0 * eps * fabs(tau) || r.iter >= max_iter) {
        // bracket collapsed to rounding level: accept; iteration cap: flag
        if (r.iter >= max_iter && !(r.hi - r.lo <= 2.0 * eps * fabs(tau))) {
            r.failed = 1;
        }
        r.stage = 2;
        return 2;
    }

    // switching rule between fixed-weight and middle-way models
    if (!r.last) {
        if (r.iter == 2) {
            r.swtch = (r.org == r.p) ? (-w > fabs(r.prevw) * 0.1)
                                     : (w > fabs(r.prevw) * 0.1);
        } else if (r.iter > 2) {
            if (w * r.prevw > 0.0 && fabs(w) > fabs(r.prevw) * 0.1) {
                r.swtch = !r.swtch;
            }
        }
    }
    r.prevw = w;

    double eta;
    if (!r.last) {
        double c;
        if (r.swtch && r.iter > 1) {
            c = w - dlp * dpsi_f - dlq * dphi_f;
        } else if (r.org == r.p) {
            // fixed weight: (d_p - d_q) * (z_p / delta_p)^2
            c = w - dlq * dw - (r.dp - r.dq) * dtp;
        } else {
            c = w - dlp * dw - (r.dq - r.dp) * dtq;
        }
        const double a = (dlp + dlq) * w - dlp * dlq * dw;
        const double b = dlp * dlq * w;
        if (c == 0.0) {
            double aa = a;
            if (aa == 0.0) {
                if (r.swtch && r.iter > 1) {
                    aa = dlp * dlp * dpsi_f + dlq * dlq * dphi_f;
                } else if (r.org == r.p) {
                    aa = r.zp2 + dlq * dlq * dw;
                } else {
                    aa = r.zq2 + dlp * dlp * dw;
                }
            }
            eta = b * brdc_rcp(aa);
        } else if (a <= 0.0) {
            eta = (a - sqrt(fabs(a * a - 4.0 * b * c))) * brdc_rcp(2.0 * c);
        } else {
            eta = 2.0 * b * brdc_rcp(a + sqrt(fabs(a * a - 4.0 * b * c)));
        }
        if (w * eta >= 0.0) {
            eta = -w * brdc_rcp(dw);
        }
    } else {
        const double c0 = w - dlp * dpsi_f - dlq * dphi_f;
        const double c = (r.iter == 1) ? fabs(c0) : c0;
        const double a = (dlp + dlq) * w - dlp * dlq * dw;
        const double b = dlp * dlq * w;
        if (c == 0.0) {
            eta = r.hi - tau;
        } else if (a >= 0.0) {
            eta = (a + sqrt(fabs(a * a - 4.0 * b * c))) * brdc_rcp(2.0 * c);
        } else {
            eta = 2.0 * b * brdc_rcp(a - sqrt(fabs(a * a - 4.0 * b * c)));
        }
        if (w * eta > 0.0) {
            eta = -w * brdc_rcp(dw);
        }
    }
    double tnew = tau + eta;
    if (!(tnew > r.lo && tnew < r.hi)) {
        eta = (w < 0.0) ? 0.5 * (r.hi - tau) : 0.5 * (r.lo - tau);
        tnew = tau + eta;
    }
    r.tau = tnew;
    r.etau = tnew;
    r.eorg_d = r.dorg;
    return 1;
}

// Host/serial driver: solve root i of (d, z, rho) with K >= 1 poles by
// repeated full sweeps.  Returns the number of sweeps; *org/*tau describe
// the root (lambda = d[*org] + *tau).  Used by the CPU unit tests only.
__host__ __device__ inline int sec_solve_serial(int K, const double *d,
                                                const double *z, double rho,
                                                double znorm2, int i, int *org,
                                                double *tau, int *failed,
                                                double eps, int max_iter = kSecularMaxIter) {
    if (K == 1) {
        *org = 0;
        *tau = rho * z[0] * z[0];
        *failed = 0;
        return 0;
    }
    SecRoot r;
    sec_init(r, i, K, d, z, rho, znorm2);
    int sweeps = 0;
    while (r.stage != 2) {
        SecSums s;
        sec_zero(s);
        for (int j = 0; j < K; ++j) {
            sec_accum(s, r, j, d[j], z[j]);
        }
        ++sweeps;
        sec_after_sweep(r, s, eps, max_iter);
    }
    *org = r.org;
    *tau = r.tau;
    *failed = r.failed;
    return sweeps;
}

} // namespace brdc
