// brdc_backward.cuh -- adjoint of the BR solve (no counterpart in the
// reference, whose solver is values only).
//
// For L = sum_i G_i * lambda_i the solve is reverse-differentiated merge by
// merge, from the instance roots down to the leaves, using the per-level
// state the forward solve recorded in a checkpointing workspace.  Nothing
// of size n x n is formed: every merge is the map
//   (child spectra, child first/last rows, beta = |E_cut|)
//      -> (merged spectrum, merged first/last rows),
// and its adjoint needs only O(K^2) sums over pole-root pairs.
//
// One merge (poles d, weights z, rows f, l, rho = 2 beta, roots lambda_j,
// delta_ij = d_i - lambda_j computed from the compact (origin, tau) pair):
//   secular equation  1/rho + sum_i z_i^2 / delta_ij = 0   (implicit
//   function theorem: dlambda_j/dd_i = z_i^2/(delta^2 S2_j),
//   dlambda_j/dz_i = -2 z_i/(delta S2_j), dlambda_j/drho = 1/(rho^2 S2_j),
//   S2_j = sum_i z_i^2/delta_ij^2)
//   new rows  f'_j = a_j / sqrt(S2_j),  a_j = sum_i f_i z_i / delta_ij
//             (l' likewise), z taken as the Loewner value w.
// Per root the adjoint needs six sums over the poles (k_bw_roots), per pole
// four sums over the roots (k_bw_poles), written pair by pair so that a
// root lying within z_o^2 of its origin pole o costs no cancellation.  Deflation is undone by reversing
// each Givens chain (k_bw_undeflate), the merge permutation by a gather;
// the leaves by the eigenvector adjoint of their 16x16 Jacobi solve
// (k_bw_leaf).  d(L)/dE at a cut collects 2*sign(E)*dL/drho from its merge
// and -sign(E)*dL/dD' from the two leaf corners the cut modified
// (k_bw_cuts), in a fixed order, so the adjoint is bitwise reproducible.
#pragma once

#include "brdc_kernels.cuh"

namespace brdc {

struct BArgs {
    Forest F;
    Ws w;
    const double *D;
    const double *E;
    const double *G;   // dL/dW
    double *gD;
    double *gE;
    int k;
    int nodes;
    long long level_rows; // rows of the instances merging at this level
    int lanes_target;     // threads the per-row sweeps aim to keep busy
};

__device__ inline double sgn(double x) { return (double)((x > 0.0) - (x < 0.0)); }

// ---------------------------------------------------------------- unplace
// The inverse of k_place: the cotangent of every slot of a merged node
// (root, small-z deflated, rotated out) is read from its place in the
// node's ascending order.  Instance roots read dL/dW and have no row
// cotangents.
__global__ void __launch_bounds__(256) k_bw_unplace(BArgs a, long long total_n) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    const Ws &w = a.w;
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < total_n;
         x += (long long)gridDim.x * blockDim.x) {
        int g, m, depth;
        long long gs;
        if (!elem_node(a.F, a.k, x, &g, &gs, &m, &depth)) {
            continue;
        }
        const long long po = (gs + g + 1) & ~1LL;
        const int s = (int)(x - gs);
        const int K = w.nK[g];
        const int Kz = w.nKz[g];
        const int ndz = m - Kz, ndg = Kz - K;
        const bool top = (depth == 0);
        const double *zdl = w.zd + gs;
        const double *gdl = w.gd + gs;
        const double *rl = w.rlam + po;
        double val;
        int pos;
        if (s < K) {
            val = rl[s];
            pos = s + lower_bound_d(zdl, ndz, val) + lower_bound_d(gdl, ndg, val);
        } else if (s < K + ndz) {
            const int q = s - K;
            val = zdl[q];
            pos = q + upper_bound_d(rl, K, val) + lower_bound_d(gdl, ndg, val);
        } else {
            const int q = s - K - ndz;
            val = gdl[q];
            pos = q + upper_bound_d(rl, K, val) + upper_bound_d(zdl, ndz, val);
        }
        const long long o = gs + pos;
        const double cm = top ? a.G[o] : w.bnd[o];
        const double cf = top ? 0.0 : w.bnf[o];
        const double cl = top ? 0.0 : w.bnl[o];
        if (s < K) {
            w.blam[po + s] = cm;
            w.bfr[po + s] = cf;
            w.blr[po + s] = cl;
        } else if (s < K + ndz) {
            const int q = s - K;
            w.bzd[gs + q] = cm;
            w.bzf[gs + q] = cf;
            w.bzl[gs + q] = cl;
        } else {
            const int q = s - K - ndz;
            w.bgd[gs + q] = cm;
            w.bgf[gs + q] = cf;
            w.bgl[gs + q] = cl;
        }
    }
}

// Warp work items of the sweep phases: the forward plan's warp items, then
// each CTA item split into 8 warp items (same lanes per root).
struct WarpItem {
    int g;
    int first; // first root / pole of the item
    int tpr;
    int count; // roots / poles of the item
};

__device__ inline bool warp_item(const Ws &w, const LevelCtl *ctl, int wi, WarpItem *it) {
    const int iw = ctl->items_w;
    if (wi < iw) {
        it->g = w.items_w[wi];
        it->tpr = ctl->tpr_w;
        it->count = 32 / it->tpr;
        it->first = (wi - w.pref_w[it->g]) * it->count;
        return true;
    }
    const int ci = (wi - iw) >> 3, sub = (wi - iw) & 7;
    if (ci >= ctl->items_c) {
        return false;
    }
    it->g = w.items_c[ci];
    it->tpr = ctl->tpr_c;
    it->count = 32 / it->tpr;
    const int R = kSweepThreads / it->tpr;
    it->first = (ci - w.pref_c[it->g]) * R + sub * it->count;
    return true;
}

// ------------------------------------------------------------ root sums
// Root j with origin pole o (delta_oj = -tau_j), eigenvector entries
// u_i = z_i / (delta_i N), N^2 = S2 = sum z_i^2/delta_i^2, new rows
// f' = sum f_i u_i, l' = sum l_i u_i.  Every pole-root pair contributes
//   dd_i: kappa u_i^2 - (u_i/delta_i) (gf (f_i - f' u_i) + gl (l_i - l' u_i))
//   dz_i: (1/N) ((gf (f_i - f' u_i) + gl (l_i - l' u_i))/delta_i - 2 u_i kappa)
//   df_i: gf u_i,  dl_i: gl u_i,  drho: kappa / (rho^2 S2)
// with kappa = glam + gf Phi_f + gl Phi_l, Phi_f = sum u_i (f_i - f' u_i)/delta_i
// (the derivative of f' along lambda).  When z_o is small the root hugs
// its origin (|delta_o| ~ z_o^2), u_o ~ 1 and the origin terms are each of
// size 1/|delta_o| while their sum is O(1); so this kernel sums over the
// poles other than o and forms the origin's terms from those partial sums
// with 1 - u_o^2 = S_x = sum_{i != o} u_i^2 and
//   f_o - f' u_o = f_o S_x - u_o sum_{i != o} f_i u_i,
// which cancels nothing.  Per root it stores 1/N, h = gf f' + gl l', kappa,
// the origin's dd and dz terms for the pole kernel and its drho term, which
// k_bw_undeflate sums in a fixed order.
__global__ void __launch_bounds__(kSweepThreads) k_bw_roots(BArgs a) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    const Ws &w = a.w;
    const LevelCtl *ctl = &w.hdr->lvl[a.k];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = ctl->items_w + 8 * ctl->items_c;
    for (int wi = blockIdx.x * kWarpsPerBlock + warp; wi < total;
         wi += gridDim.x * kWarpsPerBlock) {
        WarpItem it;
        if (!warp_item(w, ctl, wi, &it)) {
            break;
        }
        const NodeGeom G = node_geom(a.F, a.k, it.g);
        const int K = w.nK[it.g];
        const long long po = G.poff;
        const bool top = (G.depth == 0);
        const int tpr = it.tpr;
        const int grp = lane / tpr, l = lane % tpr;
        const int j = it.first + grp;
        const bool act = (grp < it.count) && (j < K);
        const double *zz = top ? w.pz + po : w.pw + po;
        const double *pd = w.pd + po;
        const double *pf = w.pf + po;
        const double *pl = w.pl + po;
        // sums over i != o: S2x = sum u'^2, S3x = sum u'^2/delta, ax = sum f u',
        // bx = sum l u', A2x = sum f u'/delta, B2x = sum l u'/delta (u' = z/delta)
        double S2x = 0.0, S3x = 0.0, ax = 0.0, bx = 0.0, A2x = 0.0, B2x = 0.0;
        double dorg = 0.0, tau = 0.0;
        int o = -1;
        if (act) {
            o = w.rorg[po + j];
            dorg = w.rdo[po + j];
            tau = w.rtau[po + j];
            for (int i = l; i < K; i += tpr) {
                if (i == o) {
                    continue;
                }
                const double r = brdc_rcp((__ldg(pd + i) - dorg) - tau);
                const double u = __ldg(zz + i) * r;
                S2x += u * u;
                S3x += u * u * r;
                if (!top) {
                    const double fi = __ldg(pf + i), li = __ldg(pl + i);
                    ax += fi * u;
                    bx += li * u;
                    A2x += fi * u * r;
                    B2x += li * u * r;
                }
            }
        }
        S2x = group_sum(S2x, tpr);
        S3x = group_sum(S3x, tpr);
        ax = group_sum(ax, tpr);
        bx = group_sum(bx, tpr);
        A2x = group_sum(A2x, tpr);
        B2x = group_sum(B2x, tpr);
        if (act && l == 0) {
            const double dlo = -tau;
            const double uo1 = zz[o] / dlo;
            const double S2 = S2x + uo1 * uo1;
            const double invn = 1.0 / sqrt(S2);
            const double uo = uo1 * invn;
            const double Sx = S2x / S2;
            double kx = w.blam[po + j], q = 0.0, h = 0.0;
            if (!top) {
                const double fo = pf[o], lo = pl[o];
                const double gf = w.bfr[po + j], gl = w.blr[po + j];
                const double fp = (ax + fo * uo1) * invn;
                const double lp = (bx + lo * uo1) * invn;
                const double nfo = fo * Sx - uo * (ax * invn);
                const double nlo = lo * Sx - uo * (bx * invn);
                q = gf * nfo + gl * nlo;
                kx += gf * (A2x * invn - fp * S3x / S2) + gl * (B2x * invn - lp * S3x / S2);
                h = gf * fp + gl * lp;
                w.rfp[po + j] = fp;
                w.rlp[po + j] = lp;
            }
            const double kap = kx + (uo / dlo) * q;
            w.rinvn[po + j] = invn;
            w.rh[po + j] = h;
            w.rkap[po + j] = kap;
            w.rcdo[po + j] = kx * uo * uo - uo * q * Sx / dlo;
            w.rczo[po + j] = (q * (Sx - uo * uo) / dlo - 2.0 * uo * kx) * invn;
            // inner merges read the Loewner weights, sqrt(rho) * z
            const double rho = w.nrho[it.g];
            w.rkr[po + j] = kap / ((top ? rho : 1.0) * rho * S2);
        }
    }
}

// ------------------------------------------------------------ pole sums
// Pole i sums the pair terms above over the roots whose origin is not i;
// the (at most two) roots j in {i-1, i} with origin i add their stored
// origin terms instead.
__global__ void __launch_bounds__(kSweepThreads) k_bw_poles(BArgs a) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    const Ws &w = a.w;
    const LevelCtl *ctl = &w.hdr->lvl[a.k];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = ctl->items_w + 8 * ctl->items_c;
    for (int wi = blockIdx.x * kWarpsPerBlock + warp; wi < total;
         wi += gridDim.x * kWarpsPerBlock) {
        WarpItem it;
        if (!warp_item(w, ctl, wi, &it)) {
            break;
        }
        const NodeGeom G = node_geom(a.F, a.k, it.g);
        const int K = w.nK[it.g];
        const long long po = G.poff;
        const bool top = (G.depth == 0);
        const int tpr = it.tpr;
        const int grp = lane / tpr, l = lane % tpr;
        const int i = it.first + grp;
        const bool act = (grp < it.count) && (i < K);
        double gd = 0.0, gz = 0.0, gF = 0.0, gL = 0.0;
        int sk0 = -1, sk1 = -1;
        double zi = 0.0, fi = 0.0, li = 0.0;
        if (act) {
            const double di = w.pd[po + i];
            zi = top ? w.pz[po + i] : w.pw[po + i];
            if (!top) {
                fi = w.pf[po + i];
                li = w.pl[po + i];
            }
            sk0 = (i > 0 && w.rorg[po + i - 1] == i) ? i - 1 : -1;
            sk1 = (w.rorg[po + i] == i) ? i : -1;
            const double *rdo = w.rdo + po;
            const double *rtau = w.rtau + po;
            const double *rin = w.rinvn + po;
            const double *rk = w.rkap + po;
            if (top) {
                for (int j = l; j < K; j += tpr) {
                    if (j == sk0 || j == sk1) {
                        continue;
                    }
                    const double r = brdc_rcp((di - __ldg(rdo + j)) - __ldg(rtau + j));
                    const double in = __ldg(rin + j);
                    const double u = zi * r * in;
                    const double kj = __ldg(rk + j);
                    gd += u * u * kj;
                    gz -= 2.0 * u * kj * in;
                }
            } else {
                const double *bf = w.bfr + po;
                const double *bl = w.blr + po;
                const double *rh = w.rh + po;
                for (int j = l; j < K; j += tpr) {
                    if (j == sk0 || j == sk1) {
                        continue;
                    }
                    const double r = brdc_rcp((di - __ldg(rdo + j)) - __ldg(rtau + j));
                    const double in = __ldg(rin + j);
                    const double u = zi * r * in;
                    const double kj = __ldg(rk + j);
                    const double gfj = __ldg(bf + j), glj = __ldg(bl + j);
                    const double q = gfj * fi + glj * li - u * __ldg(rh + j);
                    gd += u * (u * kj - q * r);
                    gz += in * (q * r - 2.0 * u * kj);
                    gF += gfj * u;
                    gL += glj * u;
                }
            }
        }
        gd = group_sum(gd, tpr);
        gz = group_sum(gz, tpr);
        gF = group_sum(gF, tpr);
        gL = group_sum(gL, tpr);
        if (act && l == 0) {
            const int sk[2] = {sk0, sk1};
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const int j = sk[t];
                if (j < 0) {
                    continue;
                }
                gd += w.rcdo[po + j];
                gz += w.rczo[po + j];
                if (!top) {
                    const double u = zi / (-w.rtau[po + j]) * w.rinvn[po + j];
                    gF += w.bfr[po + j] * u;
                    gL += w.blr[po + j] * u;
                }
            }
            w.bpd[po + i] = gd;
            // 1/N above is in the scale of the weights read; inner merges
            // read sqrt(rho) * z
            w.bpz[po + i] = top ? gz : gz * sqrt(w.nrho[it.g]);
            w.bpf[po + i] = gF;
            w.bpl[po + i] = gL;
        }
    }
}

// ------------------------------------------------------------- deflated
// The forward treats a deflated eigenvector as exact.  Its value is right to
// the deflation tolerance, but two first-order couplings between it and the
// roots' eigenvectors u_j survive, and they move the boundary rows (so inner
// merges only; at an instance root no rows are carried):
//  * small-z pole i (eigenvector e_i, weight z_i ~ 0): the rank-one term
//    rho z z^T turns e_i and u_j into each other,
//      dL/dz_i = sum_j (1/N_j)/delta_ij (gf_j f_i + gl_j l_i - gf_i f'_j - gl_i l'_j);
//  * rotated-out member m of the cluster whose final base is pole p (rows
//    f_m, l_m after the rotations): the neglected off-diagonal
//    omega = c s (d_m - d_base), zero at a tie, couples m to p,
//      dL/domega = z_p sum_j (1/N_j)/delta_pj^2
//                  (gf_m f'_j + gl_m l'_j - gf_j f_m - gl_j l_m),
//    which k_bw_undeflate turns into +-c s dL/domega on the two d's.
// `tpr` lanes per deflated row (where deflated rows are most of the level:
// enough to reach lanes_target threads, at least ~8 roots per lane on
// average); the lanes stride over the roots and combine by shuffles.  Every warp runs the same number of trips,
// so the shuffles stay convergent.
__global__ void __launch_bounds__(256) k_bw_defl(BArgs a, long long total_n) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    const Ws &w = a.w;
    const LevelCtl *ctl = &w.hdr->lvl[a.k];
    const long long ndefl = a.level_rows - ctl->total_k;
    const double kavg = (double)ctl->total_k / (double)(a.nodes > 0 ? a.nodes : 1);
    // more lanes per row only where deflated rows are most of the level:
    // below that, every extra lane mostly classifies rows that need nothing
    int tpr = 1;
    while (2 * ndefl > a.level_rows && tpr < 32 &&
           (double)tpr * (double)ndefl < (double)a.lanes_target &&
           8.0 * (double)(2 * tpr) <= kavg) {
        tpr <<= 1;
    }
    const long long slots = ((total_n * tpr + 31) / 32) * 32;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < slots; t += stride) {
        const long long x = t / tpr;
        const int l = (int)(t % tpr);
        double acc = 0.0;
        bool out = false, small = false;
        long long gs = 0, dst = 0;
        double scale = 1.0;
        int g, m, depth;
        if (x < total_n && elem_node(a.F, a.k, x, &g, &gs, &m, &depth) && depth != 0) {
            const long long po = (gs + g + 1) & ~1LL;
            const int s = (int)(x - gs);
            const int K = w.nK[g];
            const int Kz = w.nKz[g];
            const int ndz = m - Kz;
            if (s >= K) {
                small = s < K + ndz;
                const int q = small ? s - K : s - K - ndz;
                double di, fi, li, gfi, gli, zp = 1.0;
                if (small) {
                    di = w.zd[gs + q];
                    fi = w.zf[gs + q];
                    li = w.zl[gs + q];
                    gfi = w.bzf[gs + q];
                    gli = w.bzl[gs + q];
                } else {
                    const int act = w.gpos[gs + q];
                    const int p = lower_bound_int(w.pmap + po, K, w.gbase[gs + act]);
                    di = w.pd[po + p];
                    zp = w.pw[po + p];
                    fi = w.af[gs + act];
                    li = w.al[gs + act];
                    gfi = w.bgf[gs + q];
                    gli = w.bgl[gs + q];
                }
#pragma unroll 4
                for (int j = l; j < K; j += tpr) {
                    const double r = brdc_rcp((di - __ldg(w.rdo + po + j)) - __ldg(w.rtau + po + j));
                    const double tt = __ldg(w.bfr + po + j) * fi + __ldg(w.blr + po + j) * li -
                                      gfi * __ldg(w.rfp + po + j) - gli * __ldg(w.rlp + po + j);
                    acc += __ldg(w.rinvn + po + j) * r * (small ? tt : -tt * r);
                }
                out = true;
                dst = gs + q;
                // 1/N_j is in the scale of the Loewner weights, sqrt(rho) z;
                // the omega sum multiplies it by a weight of the same scale
                scale = small ? sqrt(w.nrho[g]) : zp;
            }
        }
        acc = group_sum(acc, tpr);
        if (out && l == 0) {
            if (small) {
                w.bzz[dst] = acc * scale;
            } else {
                w.bgw[dst] = scale * acc;
            }
        }
    }
}

// Reverse the rotation chain based at active index b0 of a merge (a cluster
// is a base with gmark 0 followed by its members, gmark 1, rotated in
// increasing order); false if no chain starts there.
__device__ inline bool bw_reverse_chain(const Ws &w, long long gs, int b0, int Kz) {
    if (w.gmark[gs + b0] != 0 || b0 + 1 >= Kz || w.gmark[gs + b0 + 1] == 0) {
        return false;
    }
    {
        int c = 1;
        while (b0 + c + 1 < Kz && w.gmark[gs + b0 + c + 1] != 0) {
            ++c;
        }
        double fb = w.af[gs + b0], lb = w.al[gs + b0];       // rows after the chain
        double gfb = w.baf[gs + b0], glb = w.bal[gs + b0], gzb = w.baz[gs + b0];
        double gdb = w.bad[gs + b0];
        double pic = 1.0; // product of the later rotations' c: omega_k reaches the final base scaled by it
        for (int kk = c; kk >= 1; --kk) {
            const long long x = gs + b0 + kk;
            const double cc = w.gc[x], ss = w.gs[x], rr = w.gr[x];
            const double fx2 = w.af[x], lx2 = w.al[x];          // member rows after
            const double fb1 = cc * fb - ss * fx2, fx1 = ss * fb + cc * fx2;
            const double lb1 = cc * lb - ss * lx2, lx1 = ss * lb + cc * lx2;
            const double gfx2 = w.baf[x], glx2 = w.bal[x];
            const double gfb1 = cc * gfb - ss * gfx2, gfx1 = ss * gfb + cc * gfx2;
            const double glb1 = cc * glb - ss * glx2, glx1 = ss * glb + cc * glx2;
            const double gcs = gfb * fb1 + gfx2 * fx1 + glb * lb1 + glx2 * lx1;
            const double gsn = gfb * fx1 - gfx2 * fb1 + glb * lx1 - glx2 * lb1;
            // r = hypot(zb, zx), c = zb/r, s = zx/r
            const double gzb1 = gzb * cc + (gcs * ss * ss - gsn * cc * ss) / rr;
            const double gzx = gzb * ss + (-gcs * cc * ss + gsn * cc * cc) / rr;
            // d of the rotated pair: the Rayleigh quotients c^2 d_b + s^2 d_x
            // and s^2 d_b + c^2 d_x, equal to the kept d_b, d_x up to the
            // deflation tolerance and exact at a tie, where they are the
            // derivative of the eigenvalues the deflation finds
            const double c2 = cc * cc, s2 = ss * ss, gdx2 = w.bad[x];
            const double gom = cc * ss * pic * w.baz[x];
            w.bad[x] = s2 * gdb + c2 * gdx2 + gom;
            gdb = c2 * gdb + s2 * gdx2 - gom;
            pic *= cc;
            w.baf[x] = gfx1;
            w.bal[x] = glx1;
            w.baz[x] = gzx;
            fb = fb1;
            lb = lb1;
            gfb = gfb1;
            glb = glb1;
            gzb = gzb1;
        }
        w.baf[gs + b0] = gfb;
        w.bal[gs + b0] = glb;
        w.baz[gs + b0] = gzb;
        w.bad[gs + b0] = gdb;
    }
    return true;
}

// ------------------------------------------------------------- undeflate
// One CTA per merge: pole and rotated-out cotangents back to the active
// list, each Givens chain reversed (rows and z), active and small-z lists
// back to merged positions, merged positions back to the two children
// (z = last row of the left child / first row of the right child, over
// sqrt 2), and dL/dE at the cut.
template <int T>
__global__ void __launch_bounds__(T) k_bw_undeflate(BArgs a) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    __shared__ int iscan[32];
    __shared__ double red[32];
    const int g = blockIdx.x;
    const NodeGeom G = node_geom(a.F, a.k, g);
    const Ws &w = a.w;
    const long long gs = G.gstart, po = G.poff;
    const int m = G.m, m1 = G.m1;
    const int K = w.nK[g];
    const int Kz = w.nKz[g];
    const int ndz = m - Kz;
    const bool top = (G.depth == 0);
    const double isq2 = 0.70710678118654752440;

    // poles -> active positions; rotated-out eigenvalues and rows by rank
    // among the active positions with gmark set
    for (int i = threadIdx.x; i < K; i += T) {
        const long long o = gs + w.pmap[po + i];
        w.bad[o] = w.bpd[po + i];
        w.baz[o] = w.bpz[po + i];
        w.baf[o] = w.bpf[po + i];
        w.bal[o] = w.bpl[po + i];
    }
    int carry = 0;
    for (int base = 0; base < Kz; base += T) {
        const int a0 = base + threadIdx.x;
        const int mk = (a0 < Kz) ? w.gmark[gs + a0] : 0;
        int tot;
        const int ex = block_exscan<T>(mk, iscan, &tot);
        if (mk) {
            const int q = carry + ex;
            const long long o = gs + a0;
            w.bad[o] = w.bgd[gs + q];
            // a rotated-out member's z is zero for every z, so its slot
            // carries dL/domega to the chain reversal instead
            w.baz[o] = top ? 0.0 : w.bgw[gs + q];
            w.baf[o] = w.bgf[gs + q];
            w.bal[o] = w.bgl[gs + q];
        }
        carry += tot;
    }
    __syncthreads();

    // reverse every rotation chain
    for (int b0 = threadIdx.x; b0 < Kz; b0 += T) {
        bw_reverse_chain(w, gs, b0, Kz);
    }
    double kr = 0.0;
    for (int j = threadIdx.x; j < K; j += T) {
        kr += w.rkr[po + j];
    }
    const double grho = block_sum<T>(kr, red);
    __syncthreads();

    // active and small-z lists -> merged positions
    for (int i = threadIdx.x; i < Kz; i += T) {
        const long long p = gs + w.amap[gs + i];
        w.bmd[p] = w.bad[gs + i];
        w.bmz[p] = w.baz[gs + i];
        w.bmf[p] = w.baf[gs + i];
        w.bml[p] = w.bal[gs + i];
    }
    for (int q = threadIdx.x; q < ndz; q += T) {
        const long long p = gs + w.zmap[gs + q];
        w.bmd[p] = w.bzd[gs + q];
        w.bmz[p] = top ? 0.0 : w.bzz[gs + q];
        w.bmf[p] = w.bzf[gs + q];
        w.bml[p] = w.bzl[gs + q];
    }
    __syncthreads();

    // merged positions -> children
    for (int p = threadIdx.x; p < m; p += T) {
        const long long x = gs + w.morig[gs + p];
        const int e = (int)(x - gs);
        w.bcd[x] = w.bmd[gs + p];
        if (e < m1) {
            w.bcf[x] = w.bmf[gs + p];
            w.bcl[x] = w.bmz[gs + p] * isq2;
        } else {
            w.bcf[x] = w.bmz[gs + p] * isq2;
            w.bcl[x] = w.bml[gs + p];
        }
    }
    if (threadIdx.x == 0) {
        const long long cut = gs + m1 - 1;
        a.gE[cut] = 2.0 * sgn(a.E[cut]) * grho;
    }
}

// The same undeflation for the large merges near the top, where one CTA per
// merge would stream tens of thousands of rows alone: five grid-wide passes
// over the level's rows, each row one independent gather or scatter.  The
// rotated-out slot q finds its active index through gpos, so no scan is
// needed.

// poles and rotated-out members -> active positions
__global__ void __launch_bounds__(256) k_bw_ud_active(BArgs a, long long total_n) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    const Ws &w = a.w;
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < total_n;
         x += (long long)gridDim.x * blockDim.x) {
        int g, m, depth;
        long long gs;
        if (!elem_node(a.F, a.k, x, &g, &gs, &m, &depth)) {
            continue;
        }
        const long long po = (gs + g + 1) & ~1LL;
        const int s = (int)(x - gs);
        const int K = w.nK[g], Kz = w.nKz[g];
        if (s < K) {
            const long long o = gs + w.pmap[po + s];
            w.bad[o] = w.bpd[po + s];
            w.baz[o] = w.bpz[po + s];
            w.baf[o] = w.bpf[po + s];
            w.bal[o] = w.bpl[po + s];
        } else if (s < Kz) {
            const int q = s - K;
            const long long o = gs + w.gpos[gs + q];
            w.bad[o] = w.bgd[gs + q];
            // a rotated-out member's z is zero for every z, so its slot
            // carries dL/domega to the chain reversal instead
            w.baz[o] = depth == 0 ? 0.0 : w.bgw[gs + q];
            w.baf[o] = w.bgf[gs + q];
            w.bal[o] = w.bgl[gs + q];
        }
    }
}

// Givens chains, one thread per active index (chain bases do the work)
__global__ void __launch_bounds__(256) k_bw_ud_chains(BArgs a, long long total_n) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    const Ws &w = a.w;
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < total_n;
         x += (long long)gridDim.x * blockDim.x) {
        int g, m, depth;
        long long gs;
        if (!elem_node(a.F, a.k, x, &g, &gs, &m, &depth)) {
            continue;
        }
        const int s = (int)(x - gs);
        const int Kz = w.nKz[g];
        if (s < Kz) {
            bw_reverse_chain(w, gs, s, Kz);
        }
    }
}

// active and small-z lists -> merged positions
__global__ void __launch_bounds__(256) k_bw_ud_merged(BArgs a, long long total_n) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    const Ws &w = a.w;
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < total_n;
         x += (long long)gridDim.x * blockDim.x) {
        int g, m, depth;
        long long gs;
        if (!elem_node(a.F, a.k, x, &g, &gs, &m, &depth)) {
            continue;
        }
        const int s = (int)(x - gs);
        const int Kz = w.nKz[g];
        if (s < Kz) {
            const long long p = gs + w.amap[gs + s];
            w.bmd[p] = w.bad[gs + s];
            w.bmz[p] = w.baz[gs + s];
            w.bmf[p] = w.baf[gs + s];
            w.bml[p] = w.bal[gs + s];
        } else {
            const int q = s - Kz;
            const long long p = gs + w.zmap[gs + q];
            w.bmd[p] = w.bzd[gs + q];
            w.bmz[p] = depth == 0 ? 0.0 : w.bzz[gs + q];
            w.bmf[p] = w.bzf[gs + q];
            w.bml[p] = w.bzl[gs + q];
        }
    }
}

// merged positions -> children (z = last row of the left child / first row
// of the right child, over sqrt 2)
__global__ void __launch_bounds__(256) k_bw_ud_children(BArgs a, long long total_n) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    const Ws &w = a.w;
    const double isq2 = 0.70710678118654752440;
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < total_n;
         x += (long long)gridDim.x * blockDim.x) {
        int g, m, depth;
        long long gs;
        if (!elem_node(a.F, a.k, x, &g, &gs, &m, &depth)) {
            continue;
        }
        const int p = (int)(x - gs);
        const int m1 = m >> 1;
        const long long xc = gs + w.morig[gs + p];
        const int e = (int)(xc - gs);
        w.bcd[xc] = w.bmd[x];
        if (e < m1) {
            w.bcf[xc] = w.bmf[x];
            w.bcl[xc] = w.bmz[x] * isq2;
        } else {
            w.bcf[xc] = w.bmz[x] * isq2;
            w.bcl[xc] = w.bml[x];
        }
    }
}

// dL/drho of every merge summed over its roots by one warp, in a fixed
// order, and dL/dE at its cut
__global__ void __launch_bounds__(256) k_bw_ud_rho(BArgs a) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    const Ws &w = a.w;
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long g = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < a.nodes;
         g += warps) {
        const NodeGeom G = node_geom(a.F, a.k, (int)g);
        const int K = w.nK[g];
        double kr = 0.0;
        for (int j = lane; j < K; j += 32) {
            kr += w.rkr[G.poff + j];
        }
        kr = warp_sum(kr);
        if (lane == 0) {
            const long long cut = G.gstart + G.m1 - 1;
            a.gE[cut] = 2.0 * sgn(a.E[cut]) * kr;
        }
    }
}

// ------------------------------------------------------------------ leaves
// The leaf's whole eigenvector matrix V, kept by the checkpointing forward
// (k_leaf_full, column x of V in lane x), then
//   Abar = V sym(diag(glam) + F o (V^T Vbar)) V^T,  F_kl = 1/(lambda_l -
//   lambda_k), Vbar nonzero only in rows 0 and s-1 (the boundary rows),
// gD = diag(Abar), gE = 2 sign(E) Abar_{j,j+1}, and the corner corrections
// of the cuts.
__global__ void __launch_bounds__(kLeafWarps * 32)
    k_bw_leaf(BArgs a, long long total_leaves) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    __shared__ double sV[kLeafWarps * 2][16][17];
    __shared__ double sC[kLeafWarps * 2][16][17];
    __shared__ double sLam[kLeafWarps * 2][16], sV0[kLeafWarps * 2][16], sV1[kLeafWarps * 2][16];
    __shared__ double sGf[kLeafWarps * 2][16], sGl[kLeafWarps * 2][16];
    const int lane = threadIdx.x & 31;
    const int x = lane & 15;
    const int half = lane >> 4;
    const int slot = (threadIdx.x >> 5) * 2 + half;
    const Ws &w = a.w;
    const long long pairs = (total_leaves + 1) / 2;
    for (long long pr = (long long)blockIdx.x * kLeafWarps + (threadIdx.x >> 5); pr < pairs;
         pr += (long long)gridDim.x * kLeafWarps) {
        const long long leaf = 2 * pr + half;
        const bool has = leaf < total_leaves;
        LeafGeom LG{};
        int s = 0;
        if (has) {
            LG = leaf_geom(a.F, leaf);
            s = LG.s;
        }
        // the forward's leaf (k_leaf_full): eigenvalue of rank x and its
        // eigenvector, in the scaled problem of the forward (the gradient
        // of a homogeneous map is scale-free, so nothing else changes)
        double v[16];
        double lamx = 0.0;
        if (x < s) {
            const long long o = LG.gstart + x;
            lamx = w.leafl[o];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                v[j] = w.leafv[o * 16 + j];
            }
        } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                v[j] = 0.0;
            }
        }
        const int rank = x; // stored in ascending order
        double gmu = 0.0, gf = 0.0, gl = 0.0;
        if (x < s) {
            const long long o = LG.gstart + rank;
            if (LG.top) {
                gmu = a.G[o];
            } else {
                gmu = w.bcd[o];
                gf = w.bcf[o];
                gl = w.bcl[o];
            }
        }
        const double v0 = v[0];
        double vlast = 0.0;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            vlast = (j == s - 1) ? v[j] : vlast;
        }
        sLam[slot][x] = lamx;
        sV0[slot][x] = v0;
        sV1[slot][x] = vlast;
        sGf[slot][x] = gf;
        sGl[slot][x] = gl;
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            sV[slot][r][x] = v[r];
        }
        __syncwarp();
        // column x of C = diag(gmu) + (M + M^T)/2, M_kl = F_kl (V0_k gf_l + V1_k gl_l)
        for (int k = 0; k < 16; ++k) {
            double cv = 0.0;
            if (x < s && k < s && k != x) {
                const double lk = sLam[slot][k], lx = sLam[slot][x];
                if (lk != lx) {
                    const double mkx = (sV0[slot][k] * gf + sV1[slot][k] * gl) / (lx - lk);
                    const double mxk = (sV0[slot][x] * sGf[slot][k] + sV1[slot][x] * sGl[slot][k]) /
                                       (lk - lx);
                    cv = 0.5 * (mkx + mxk);
                }
            } else if (k == x) {
                cv = gmu;
            }
            sC[slot][k][x] = cv;
        }
        __syncwarp();
        // row x of Abar: Abar_xx and Abar_{x,x+1}
        if (x < s) {
            double dd = 0.0, de = 0.0;
            for (int k = 0; k < s; ++k) {
                double t0 = 0.0, t1 = 0.0;
                for (int l = 0; l < s; ++l) {
                    const double ckl = sC[slot][k][l];
                    t0 += ckl * sV[slot][x][l];
                    if (x + 1 < s) {
                        t1 += ckl * sV[slot][x + 1][l];
                    }
                }
                dd += sV[slot][x][k] * t0;
                de += sV[slot][x][k] * t1;
            }
            const long long row = LG.gstart + x;
            a.gD[row] = dd;
            if (x + 1 < s) {
                a.gE[row] = 2.0 * sgn(a.E[row]) * de;
            }
        }
        __syncwarp();
    }
}

// Each cut's corner rows D'[c] = D[c] - |E_c| and D'[c+1] = D[c+1] - |E_c|:
// dL/dE_c -= sign(E_c) (dL/dD[c] + dL/dD[c+1]), on top of the merge's
// 2 sign(E_c) dL/drho stored by k_bw_undeflate.  One thread per leaf (the
// leaf left of the cut), so the sum has a fixed order.
__global__ void __launch_bounds__(256) k_bw_cuts(BArgs a, long long total_leaves) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    for (long long leaf = (long long)blockIdx.x * blockDim.x + threadIdx.x; leaf < total_leaves;
         leaf += (long long)gridDim.x * blockDim.x) {
        const LeafGeom LG = leaf_geom(a.F, leaf);
        const long long c = LG.gstart + LG.s - 1;
        if (LG.gstart + LG.s < LG.iend) {
            a.gE[c] -= sgn(a.E[c]) * (a.gD[c] + a.gD[c + 1]);
        }
    }
}

__global__ void k_bw_zero(double *p, long long n) {
    pdl_begin();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        p[i] = 0.0;
    }
}

} // namespace brdc
