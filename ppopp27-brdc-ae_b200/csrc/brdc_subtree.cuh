// brdc_subtree.cuh -- the bottom of the merge tree in one kernel.
//
// Near the leaves the merges are small (tens to a few hundred rows) and
// numerous, so the per-level kernels spend their time on launches, global
// round trips and tails rather than arithmetic.  Here one CTA takes a whole
// subtree of at most kSubRows rows -- its leaves and its lowest kSubLevels
// merge levels -- and keeps every array of it in shared memory.  Each level
// runs the same steps as the per-level kernels, with the same rules:
//   rank merge of the two children; tolerance tol = 8 eps max(max|d|,
//   max|z|); small-z compaction (merged order kept); close-pole Givens
//   chains; pole compaction; secular roots by the state machine of
//   brdc_secular.cuh (rounds over the live roots, then one warp per root
//   for the slow tail); Loewner weights; first/last boundary rows;
//   placement in ascending order.
// Only the order of a few floating-point sums differs (sum z^2 by warp
// partials, the secular sweeps by the lanes a round gives each root), so
// deflation is decided exactly as the per-level path decides it.  In
// checkpoint mode the leaves come from k_leaf_full, and every fused level's
// state is also written to its workspace slice, in the layout the per-level
// kernels use, for the adjoint.
#pragma once

#include "brdc_kernels.cuh"

namespace brdc {

constexpr int kSubMaxLevels = 5; // merge levels a subtree can hold (leaves <= 16 rows)

// Rows (and threads) of a subtree CTA holding `levels` merge levels: a node
// of level k spans at most 2^(k+1) leaves of at most 16 rows.
constexpr int sub_rows_for(int levels) { return levels <= 4 ? 256 : 512; }

struct SubArgs {
    KArgs a;                  // forest, workspace, D, E, W, diagnostics
    Ws lw[kSubMaxLevels];     // workspace view of each fused level (checkpoint slices)
    double *out_d, *out_f, *out_l; // inputs of the first per-level merge
    int levels;               // fused merge levels (1..kSubMaxLevels)
    int ckpt;                 // write each fused level's state for the adjoint
    int leaves_done;          // the leaves were solved by k_leaf_full: read them
};

// Roots per warp at most in the barrier-free tail of the subtree's secular
// rounds (the rounds stop once the live roots fit this many per warp).
// Measured on B200 (uniform 65,536): 1 -> 0.846 ms, 4 -> 0.856, 8 -> 0.865,
// 16 -> 0.914: repacking the live roots every round beats iterating
// several of them per warp, whose lanes idle once their root converges.
#ifndef BRDC_SUB_TAIL_ROOTS
#define BRDC_SUB_TAIL_ROOTS 1
#endif
constexpr int kSubTailRoots = BRDC_SUB_TAIL_ROOTS;

template <int kSubRows>
struct SubSmem {
    static constexpr int kSubWarps = kSubRows / 32;
    double cd[kSubRows], cf[kSubRows], cl[kSubRows];   // children (sorted) / placed output
    double md[kSubRows], mz[kSubRows], mf[kSubRows], ml[kSubRows];
    double ad[kSubRows], az[kSubRows], af[kSubRows], al[kSubRows];
    double zd[kSubRows], zf[kSubRows], zl[kSubRows];
    double gd[kSubRows], gf[kSubRows], gl[kSubRows];
    double pd[kSubRows], pz[kSubRows], pf[kSubRows], pl[kSubRows], pw[kSubRows];
    double rdo[kSubRows], rtau[kSubRows], rlam[kSubRows], rf[kSubRows], rl[kSubRows];
    int morig[kSubRows], amap[kSubRows], zmap[kSubRows], gmark[kSubRows];
    int gbase[kSubRows], gpos[kSubRows], pmap[kSubRows], rorg[kSubRows];
    int ex[kSubRows + 1];
    double part[kSubWarps][kSubRows / 16];
    int nstart[kSubRows / 16], nsize[kSubRows / 16], nK[kSubRows / 16], nKz[kSubRows / 16];
    int kpre[kSubRows / 16 + 1]; // prefix of nK: roots of the level before node j
    double nrho[kSubRows / 16], ntol[kSubRows / 16], nzn[kSubRows / 16], nmaxd[kSubRows / 16];
    double nrinv[kSubRows / 16]; // 1 / rho of node j
    SecDyn dyn[kSubRows];      // parked secular state of each root between rounds
    int aq[2][kSubRows];       // unconverged roots (root | node << 16), ping-pong
    int scan[32];
    int qc[3];                 // list counters, rotating
    int it_sum, it_max, it_failed;
};

// Exclusive scan of one int per thread over the CTA; ex[kSubRows] = total.
template <int kSubRows>
__device__ inline void sub_scan(SubSmem<kSubRows> &S, int v) {
    int tot;
    const int e = block_exscan<kSubRows>(v, S.scan, &tot);
    S.ex[threadIdx.x] = e;
    if (threadIdx.x == 0) {
        S.ex[kSubRows] = tot;
    }
    __syncthreads();
}

// Per-node reduction (sum or max) of one value per row, in a fixed order:
// warp partials per node, then the warps in order.  j = node of the row
// (-1 for none); returns the node's result to threads j < nk via *out.
template <bool MAX, int kSubRows>
__device__ inline void sub_node_reduce(SubSmem<kSubRows> &S, double v, int j, int nk,
                                       double *out) {
    constexpr int kSubWarps = kSubRows / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = threadIdx.x; q < kSubWarps * (kSubRows / 16); q += kSubRows) {
        (&S.part[0][0])[q] = 0.0;
    }
    __syncthreads();
    const int jlo = __shfl_sync(kFull, j, 0);
    int jhi = j;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        jhi = max(jhi, __shfl_xor_sync(kFull, jhi, o));
    }
    for (int jj = max(jlo, 0); jj <= jhi; ++jj) {
        double t = (j == jj) ? v : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double u = __shfl_xor_sync(kFull, t, o);
            t = MAX ? fmax(t, u) : t + u;
        }
        if (lane == 0) {
            S.part[warp][jj] = t;
        }
    }
    __syncthreads();
    if (threadIdx.x < nk) {
        double r = 0.0;
        for (int w = 0; w < kSubWarps; ++w) {
            r = MAX ? fmax(r, S.part[w][threadIdx.x]) : r + S.part[w][threadIdx.x];
        }
        *out = r;
    }
    __syncthreads();
}

template <int kSubRows>
__device__ inline int sub_node_of(const SubSmem<kSubRows> &S, int nk, int x) {
    for (int j = 0; j < nk; ++j) {
        if (x < S.nstart[j] + S.nsize[j]) {
            return x >= S.nstart[j] ? j : -1;
        }
    }
    return -1;
}

template <int kSubRows>
__global__ void __launch_bounds__(kSubRows, 512 / kSubRows) k_subtree(SubArgs A) {
    pdl_begin();
    if (halted(A.a.w.hdr)) {
        return;
    }
    constexpr int kSubWarps = kSubRows / 32;
    extern __shared__ __align__(16) unsigned char sub_raw[];
    SubSmem<kSubRows> &S = *reinterpret_cast<SubSmem<kSubRows> *>(sub_raw);
    const KArgs &a = A.a;
    const Forest &F = a.F;
    const int x = threadIdx.x;
    const int warp = x >> 5, lane = x & 31;
    const double eps = DBL_EPSILON;
    const int max_iter = a.w.hdr->max_iter;

    // subtree -> instance, its levels and rows
    int b = 0;
    long long t = blockIdx.x;
    long long base = 0, n = F.n0;
    int L = F.L0;
    if (F.B > 1) {
        b = upper_bound_int(F.sub_prefix, F.B + 1, (int)blockIdx.x) - 1;
        t = blockIdx.x - F.sub_prefix[b];
        base = F.off[b];
        n = F.off[b + 1] - base;
        L = F.lev[b];
    }
    const int Ls = L < A.levels ? L : A.levels; // merge levels in this subtree
    const bool inst_top = (Ls == L);            // its root is the instance root
    long long sst, ssz;
    walk_node(n, L - Ls, t, &sst, &ssz);
    const long long gsub = base + sst;
    const int R = (int)ssz;
    const double esc = inst_scale(a.w, b);     // E (and D) of the scaled problem
    const double wsc = inst_unscale(a.w, b);   // back to the caller's scale

    if (x == 0) {
        S.it_sum = 0;
        S.it_max = 0;
        S.it_failed = 0;
    }

    // ---------------------------------------------------------- leaves
    if (A.leaves_done) {
        // solved by k_leaf_full (checkpointing forward): this subtree's
        // rows, sorted per leaf with their first and last rows (a one-leaf
        // instance is already in W)
        for (int r = x; r < R; r += kSubRows) {
            S.cd[r] = a.w.cd[gsub + r];
            S.cf[r] = a.w.cf[gsub + r];
            S.cl[r] = a.w.cl[gsub + r];
        }
    } else {
        int sweeps_max = 0, sweeps_sum = 0;
        const int nleaves = 1 << Ls;
        const int xl = lane & 15, half = lane >> 4;
        for (int p0 = 2 * warp; p0 < nleaves; p0 += 2 * kSubWarps) {
            const int leaf = p0 + half;
            LeafGeom LG{};
            int s = 0;
            if (leaf < nleaves) {
                long long lst, lsz;
                walk_node(R, Ls, leaf, &lst, &lsz);
                LG.gstart = gsub + lst;
                LG.istart = base;
                LG.iend = base + n;
                LG.s = (int)lsz;
                LG.top = (L == 0);
                LG.inst = b;
                s = LG.s;
            }
            double key, v0, v1;
            const int sw = leaf_solve(a, LG, s, xl, &key, &v0, &v1);
            sweeps_max = sweeps_max > sw ? sweeps_max : sw;
            sweeps_sum += (xl == 0 && s > 0) ? sw : 0;
            if (xl < s) {
                const int o = (int)(LG.gstart - gsub) + xl;
                if (LG.top) {
                    a.W[LG.gstart + xl] = key * wsc;
                } else {
                    S.cd[o] = key;
                    S.cf[o] = v0;
                    S.cl[o] = v1;
                }
            }
        }
        sweeps_sum = __reduce_add_sync(kFull, sweeps_sum);
        if (lane == 0 && sweeps_max > 0) {
            atomicMax(&a.w.hdr->leaf_sweeps_max, sweeps_max);
            atomicAdd(&a.w.hdr->leaf_sweeps_sum, sweeps_sum);
        }
    }
    __syncthreads();

    // ---------------------------------------------------------- levels
    for (int k = 0; k < Ls; ++k) {
        const Ws &lw = A.lw[k];
        const int nk = 1 << (Ls - 1 - k);
        const bool top = inst_top && (k == Ls - 1);
        if (x < nk) {
            long long st, sz;
            walk_node(R, Ls - 1 - k, x, &st, &sz);
            S.nstart[x] = (int)st;
            S.nsize[x] = (int)sz;
        }
        __syncthreads();
        const int j = x < R ? sub_node_of(S, nk, x) : -1;
        const int s = j >= 0 ? S.nstart[j] : 0;
        const int m = j >= 0 ? S.nsize[j] : 0;
        const int m1 = m >> 1;
        // global node index of node j at forest level k, and its rows
        const long long gk = (F.B > 1 ? F.node_prefix[(size_t)k * (F.B + 1) + b] : 0) +
                             t * (long long)nk;

        // merge: rank merge of the two sorted children (left wins ties)
        if (j >= 0) {
            const int e = x - s;
            const double v = S.cd[x];
            int pos;
            double z, f, l;
            if (e < m1) {
                pos = e + lower_bound_d(S.cd + s + m1, m - m1, v);
                z = S.cl[x] / kSqrt2;
                f = S.cf[x];
                l = 0.0;
            } else {
                pos = (e - m1) + upper_bound_d(S.cd + s, m1, v);
                z = S.cf[x] / kSqrt2;
                f = 0.0;
                l = S.cl[x];
            }
            S.md[s + pos] = v;
            S.mz[s + pos] = z;
            S.mf[s + pos] = f;
            S.ml[s + pos] = l;
            S.morig[s + pos] = e;
        }
        if (x < nk) {
            const int s0 = S.nstart[x], mm = S.nsize[x], h = mm >> 1;
            S.nrho[x] = 2.0 * esc * fabs(a.E[gsub + s0 + h - 1]);
            S.nmaxd[x] = fmax(fmax(fabs(S.cd[s0]), fabs(S.cd[s0 + h - 1])),
                              fmax(fabs(S.cd[s0 + h]), fabs(S.cd[s0 + mm - 1])));
        }
        __syncthreads();

        // tolerance
        {
            double mzx = 0.0;
            sub_node_reduce<true, kSubRows>(S, j >= 0 ? fabs(S.mz[x]) : 0.0, j, nk, &mzx);
            if (x < nk) {
                S.ntol[x] = kDeflTolScale * eps * fmax(S.nmaxd[x], mzx);
            }
            __syncthreads();
        }
        const double rho = j >= 0 ? S.nrho[j] : 0.0;
        const double tol = j >= 0 ? S.ntol[j] : 0.0;

        // compaction 1: small-z survivors and small-z deflated, merged order
        const bool act1 = j >= 0 && fabs(rho * S.mz[x]) > tol;
        sub_scan(S, act1 ? 1 : 0);
        const int Kz = j >= 0 ? S.ex[s + m] - S.ex[s] : 0;
        if (j >= 0) {
            const int ra = S.ex[x] - S.ex[s];
            if (act1) {
                S.ad[s + ra] = S.md[x];
                S.az[s + ra] = S.mz[x];
                S.af[s + ra] = S.mf[x];
                S.al[s + ra] = S.ml[x];
                S.amap[s + ra] = x - s;
                S.gmark[s + ra] = 0;
            } else {
                const int rz = (x - s) - ra;
                S.zd[s + rz] = S.md[x];
                S.zf[s + rz] = S.mf[x];
                S.zl[s + rz] = S.ml[x];
                S.zmap[s + rz] = x - s;
            }
        }
        if (x < nk) {
            S.nKz[x] = S.ex[S.nstart[x] + S.nsize[x]] - S.ex[S.nstart[x]];
        }
        __syncthreads();

        // close-pole Givens chains (one thread per chain start)
        if (j >= 0 && x - s < Kz) {
            const int i = x - s;
            double *ad = S.ad + s, *az = S.az + s, *af = S.af + s, *al = S.al + s;
            const double di = ad[i];
            const bool nxt = (i + 1 < Kz) && (ad[i + 1] - di <= tol);
            const bool prv = (i > 0) && (di - ad[i - 1] <= tol);
            if (nxt && !prv) {
                const long long gs = gsub + s;
                int bi = i;
                double dbase = di;
                double zb = az[i], fb = af[i], lb = al[i];
                int y = i + 1;
                double dprev = di;
                while (y < Kz) {
                    const double dy = ad[y];
                    if (!(dy - dprev <= tol)) {
                        break;
                    }
                    dprev = dy;
                    if (dy - dbase > tol) {
                        az[bi] = zb;
                        af[bi] = fb;
                        al[bi] = lb;
                        bi = y;
                        dbase = dy;
                        zb = az[y];
                        fb = af[y];
                        lb = al[y];
                        ++y;
                        continue;
                    }
                    double c, sn, r;
                    lartg(zb, az[y], &c, &sn, &r);
                    const double fy = af[y], ly = al[y];
                    af[y] = -sn * fb + c * fy;
                    al[y] = -sn * lb + c * ly;
                    fb = c * fb + sn * fy;
                    lb = c * lb + sn * ly;
                    zb = r;
                    az[y] = 0.0;
                    S.gmark[s + y] = 1;
                    S.gbase[s + y] = bi;
                    if (A.ckpt) {
                        lw.gc[gs + y] = c;
                        lw.gs[gs + y] = sn;
                        lw.gr[gs + y] = r;
                    }
                    ++y;
                }
                az[bi] = zb;
                af[bi] = fb;
                al[bi] = lb;
            }
        }
        __syncthreads();

        // compaction 2: poles and rotated-out members, active order
        const bool inact = j >= 0 && x - s < Kz;
        const bool pole = inact && S.gmark[x] == 0;
        sub_scan(S, pole ? 1 : 0);
        const int K = j >= 0 ? S.ex[s + m] - S.ex[s] : 0;
        if (inact) {
            const int i = x - s;
            const int rp = S.ex[x] - S.ex[s];
            if (pole) {
                S.pd[s + rp] = S.ad[x];
                S.pz[s + rp] = S.az[x];
                S.pf[s + rp] = S.af[x];
                S.pl[s + rp] = S.al[x];
                S.pmap[s + rp] = i;
            } else {
                const int rg = i - rp;
                S.gd[s + rg] = S.ad[x];
                S.gf[s + rg] = S.af[x];
                S.gl[s + rg] = S.al[x];
                S.gpos[s + rg] = i;
            }
        }
        {
            double zsum = 0.0;
            sub_node_reduce<false, kSubRows>(S, pole ? S.az[x] * S.az[x] : 0.0, j, nk, &zsum);
            if (x < nk) {
                S.nK[x] = S.ex[S.nstart[x] + S.nsize[x]] - S.ex[S.nstart[x]];
                S.nzn[x] = zsum;
            }
            __syncthreads();
        }

        // Secular roots in rounds of one sweep.  After every round the
        // unconverged roots are packed into a list and spread over the CTA
        // with `tpr` lanes each (the largest power of two that fits), so no
        // warp keeps iterating for one slow root while its other lanes idle,
        // and the last few roots get whole warps.  A root's state is parked
        // in shared memory between rounds.  Its arithmetic depends only on
        // tpr (which lanes take which poles), not on where the root sits in
        // the list, so the result is deterministic.  The Loewner weights and
        // boundary rows use the same spread over the poles / roots.
        if (x == 0) {
            int acc = 0;
            for (int q = 0; q < nk; ++q) {
                S.kpre[q] = acc;
                acc += S.nK[q];
            }
            S.kpre[nk] = acc;
            S.qc[0] = 0;
            S.qc[1] = 0;
            S.qc[2] = 0;
        }
        if (x < nk) {
            S.nrinv[x] = 1.0 / S.nrho[x];
        }
        __syncthreads();
        const int nroots = S.kpre[nk];
        auto root_node = [&](int id) {
            int q = 0;
            while (S.kpre[q + 1] <= id) {
                ++q;
            }
            return q;
        };
        bool multi = false;
        int myq = 0;
        if (x < nroots) {
            const int q = root_node(x);
            myq = q;
            const int rr = x - S.kpre[q], Kr = S.nK[q], sr = S.nstart[q];
            const double *pd = S.pd + sr, *pz = S.pz + sr;
            if (Kr == 1) {
                S.rorg[sr] = 0;
                S.rdo[sr] = pd[0];
                S.rtau[sr] = S.nrho[q] * pz[0] * pz[0];
                S.rlam[sr] = pd[0] + S.rtau[sr];
            } else {
                SecRoot st;
                sec_init(st, rr, Kr, pd, pz, S.nrho[q], S.nzn[q]);
                sec_park(st, S.dyn[x]);
                multi = true;
            }
        }
        sub_scan(S, multi ? 1 : 0);
        if (multi) {
            S.aq[0][S.ex[x]] = x | (myq << 16);
        }
        int nact = S.ex[kSubRows];
        int cur = 0, round = 0;
        __syncthreads();
        while (nact > 0) {
            if (nact <= kSubWarps * kSubTailRoots) {
                // The last roots (the slow tail of the iteration): R per
                // warp (the smallest power of two that covers them, dealt
                // round robin over the warps), 32 / R lanes each, iterated
                // to convergence with no barrier, parking or list between
                // sweeps.  A lane group's lanes hold the same state (the
                // butterfly sums are bit-identical); the warp loops until
                // its last root converges, and the iteration cap ends it.
                int R = 1;
                while (R < kSubTailRoots && R * kSubWarps < nact) {
                    R <<= 1;
                }
                const int lanes = 32 / R;
                const int sub = lane / lanes, l2 = lane & (lanes - 1);
                const int slot = sub * kSubWarps + (x >> 5);
                const bool act = slot < nact;
                const int code = act ? S.aq[cur][slot] : 0;
                const int id = code & 0xffff, q = code >> 16;
                const int rr = id - S.kpre[q], Kr = S.nK[q], sr = S.nstart[q];
                const double *pd = S.pd + sr, *pz = S.pz + sr;
                SecRoot st;
                if (act) {
                    sec_init_static(st, rr, Kr, pd, pz, S.nrho[q], S.nrinv[q], S.nzn[q]);
                    sec_unpark(st, S.dyn[id]);
                } else {
                    st.stage = 2;
                }
                const int pmin = rr < Kr - 2 ? rr : Kr - 2;
                for (;;) {
                    SecSums sum;
                    sec_zero(sum);
                    const bool live = act && st.stage != 2;
                    if (live) {
                        secular_span(sum, st, 0, Kr, l2, lanes, pmin, rr + 1,
                                     [&](int u, double *du, double *zu) {
                                         *du = pd[u];
                                         *zu = pz[u];
                                     });
                    }
                    sums_reduce(sum, lanes);
                    if (live) {
                        sec_after_sweep(st, sum, eps, max_iter);
                    }
                    if (__all_sync(0xffffffffu, !act || st.stage == 2)) {
                        break;
                    }
                }
                if (act && l2 == 0) {
                    sec_park(st, S.dyn[id]);
                }
                __syncthreads();
                break;
            }
            int lg = 0;
            while (lg < 5 && nact << (lg + 1) <= kSubRows) {
                ++lg;
            }
            const int tp = 1 << lg;
            const int g2 = x >> lg, l2 = x & (tp - 1);
            const bool act = g2 < nact;
            const int code = act ? S.aq[cur][g2] : 0;
            const int id = code & 0xffff, q = code >> 16;
            const int rr = id - S.kpre[q], Kr = S.nK[q], sr = S.nstart[q];
            const double *pd = S.pd + sr, *pz = S.pz + sr;
            SecRoot st;
            if (act) {
                sec_init_static(st, rr, Kr, pd, pz, S.nrho[q], S.nrinv[q], S.nzn[q]);
                sec_unpark(st, S.dyn[id]);
            } else {
                st.stage = 2;
            }
            SecSums sum;
            sec_zero(sum);
            if (act) {
                const int pmin = rr < Kr - 2 ? rr : Kr - 2;
                secular_span(sum, st, 0, Kr, l2, tp, pmin, rr + 1,
                             [&](int u, double *du, double *zu) {
                                 *du = pd[u];
                                 *zu = pz[u];
                             });
            }
            sums_reduce(sum, tp);
            if (act) {
                sec_after_sweep(st, sum, eps, max_iter);
            }
            // one barrier per round: round r appends to qc[r % 3], and
            // qc[(r+2) % 3], last read in round r-1, is cleared after this
            // round's barrier, a barrier before its next appends
            int *cnt = &S.qc[round % 3];
            const bool lead = act && l2 == 0;
            if (lead) {
                sec_park(st, S.dyn[id]);
            }
            const bool more = lead && st.stage != 2;
            const unsigned mb = __ballot_sync(0xffffffffu, more);
            int at = 0;
            if (lane == 0 && mb != 0u) {
                at = atomicAdd(cnt, __popc(mb));
            }
            at = __shfl_sync(0xffffffffu, at, 0);
            if (more) {
                S.aq[cur ^ 1][at + __popc(mb & ((1u << lane) - 1u))] = code;
            }
            __syncthreads();
            nact = *cnt;
            if (x == 0) {
                S.qc[(round + 2) % 3] = 0;
            }
            cur ^= 1;
            ++round;
        }
        // results and iteration counts, one thread per root
        {
            bool mine = false;
            int it = 0, fl = 0;
            if (x < nroots) {
                const int q = root_node(x);
                const int sr = S.nstart[q];
                if (S.nK[q] >= 2) {
                    const SecDyn &dq = S.dyn[x];
                    const int rr = x - S.kpre[q];
                    S.rorg[sr + rr] = dq.org;
                    S.rdo[sr + rr] = dq.dorg;
                    S.rtau[sr + rr] = dq.tau;
                    S.rlam[sr + rr] = dq.dorg + dq.tau;
                    mine = true;
                    it = dq.iter;
                    fl = dq.failed;
                }
            }
            const unsigned full = 0xffffffffu;
            const int sum = __reduce_add_sync(full, mine ? it : 0);
            const int mx = __reduce_max_sync(full, mine ? it : 0);
            const int nf = __reduce_add_sync(full, mine ? fl : 0);
            if (lane == 0) {
                atomicAdd(&S.it_sum, sum);
                atomicMax(&S.it_max, mx);
                atomicAdd(&S.it_failed, nf);
            }
        }
        __syncthreads();

        // lanes per pole / root for the Loewner weights and the rows
        int tpr = 1;
        while (tpr < 32 && nroots * tpr * 2 <= kSubRows) {
            tpr <<= 1;
        }
        const int grp = x / tpr, gl = x % tpr;
        const int jr = grp < nroots ? root_node(grp) : -1;
        const int rr = jr >= 0 ? grp - S.kpre[jr] : 0;  // pole / root index in its node
        const int Kr = jr >= 0 ? S.nK[jr] : 0;
        const int sr = jr >= 0 ? S.nstart[jr] : 0;
        const double rhor = jr >= 0 ? S.nrho[jr] : 0.0;
        const bool nodetop = top;

        if (!nodetop) {
            // Loewner weights (sqrt(rho) z), tpr lanes per pole
            {
                double prod = 1.0;
                if (jr >= 0) {
                    const int i = rr;
                    const double di = S.pd[sr + i];
                    int q = gl;
                    for (; q + tpr < Kr; q += 2 * tpr) {
                        const int q2 = q + tpr;
                        const double dl = (di - S.rdo[sr + q]) - S.rtau[sr + q];
                        const double dl2 = (di - S.rdo[sr + q2]) - S.rtau[sr + q2];
                        prod *= lowner_pair(dl, q == i ? 1.0 : di - S.pd[sr + q], dl2,
                                            q2 == i ? 1.0 : di - S.pd[sr + q2]);
                    }
                    if (q < Kr) {
                        const double dl = (di - S.rdo[sr + q]) - S.rtau[sr + q];
                        prod *= dl * brdc_rcp(q == i ? 1.0 : di - S.pd[sr + q]);
                    }
                }
                prod = group_prod(prod, tpr);
                if (jr >= 0 && gl == 0) {
                    const double zi = S.pz[sr + rr];
                    const double mag = sqrt(fmax(-prod, 0.0));
                    double wi = zi < 0.0 ? -mag : mag;
                    if (!(mag > 0.0) || !isfinite(mag)) {
                        wi = zi * sqrt(rhor);
                    }
                    S.pw[sr + rr] = wi;
                }
            }
            __syncthreads();
            // boundary rows, tpr lanes per root
            {
                double a1 = 0.0, a2 = 0.0, s2 = 0.0;
                if (jr >= 0) {
                    const double dorg = S.rdo[sr + rr], tau = S.rtau[sr + rr];
                    int i = gl;
                    for (; i + tpr < Kr; i += 2 * tpr) {
                        const int i2 = i + tpr;
                        double u, u2;
                        row_pair(S.pw[sr + i], (S.pd[sr + i] - dorg) - tau, S.pw[sr + i2],
                                 (S.pd[sr + i2] - dorg) - tau, &u, &u2);
                        s2 += u * u;
                        a1 += S.pf[sr + i] * u;
                        a2 += S.pl[sr + i] * u;
                        s2 += u2 * u2;
                        a1 += S.pf[sr + i2] * u2;
                        a2 += S.pl[sr + i2] * u2;
                    }
                    if (i < Kr) {
                        const double dl = (S.pd[sr + i] - dorg) - tau;
                        const double u = (dl != 0.0) ? S.pw[sr + i] * brdc_rcp(dl) : 0.0;
                        s2 += u * u;
                        a1 += S.pf[sr + i] * u;
                        a2 += S.pl[sr + i] * u;
                    }
                }
                s2 = group_sum(s2, tpr);
                a1 = group_sum(a1, tpr);
                a2 = group_sum(a2, tpr);
                if (jr >= 0 && gl == 0) {
                    const double nrm = sqrt(s2);
                    S.rf[sr + rr] = nrm > 0.0 ? a1 / nrm : 0.0;
                    S.rl[sr + rr] = nrm > 0.0 ? a2 / nrm : 0.0;
                }
            }
            __syncthreads();
        }

        // checkpoint slices of this level for the adjoint
        if (A.ckpt && j >= 0) {
            const long long gs = gsub + s;
            const long long g = gk + j;
            const long long po = (gs + g + 1) & ~1LL;
            const int e = x - s;
            const int ndz = m - Kz, ndg = Kz - K;
            lw.morig[gs + e] = S.morig[x];
            lw.md[gs + e] = S.md[x];
            lw.mz[gs + e] = S.mz[x];
            if (e < Kz) {
                lw.af[gs + e] = S.af[x];
                lw.al[gs + e] = S.al[x];
                lw.amap[gs + e] = S.amap[x];
                lw.gmark[gs + e] = S.gmark[x];
                lw.gbase[gs + e] = S.gbase[x];
            }
            if (e < ndz) {
                lw.zd[gs + e] = S.zd[x];
                lw.zf[gs + e] = S.zf[x];
                lw.zl[gs + e] = S.zl[x];
                lw.zmap[gs + e] = S.zmap[x];
            }
            if (e < ndg) {
                lw.gd[gs + e] = S.gd[x];
                lw.gf[gs + e] = S.gf[x];
                lw.gl[gs + e] = S.gl[x];
                lw.gpos[gs + e] = S.gpos[x];
            }
            if (e < K) {
                lw.pd[po + e] = S.pd[x];
                lw.pz[po + e] = S.pz[x];
                lw.pf[po + e] = S.pf[x];
                lw.pl[po + e] = S.pl[x];
                lw.pw[po + e] = top ? 0.0 : S.pw[x];
                lw.pmap[po + e] = S.pmap[x];
                lw.rorg[po + e] = S.rorg[x];
                lw.rdo[po + e] = S.rdo[x];
                lw.rtau[po + e] = S.rtau[x];
                lw.rlam[po + e] = S.rlam[x];
            }
            if (e == 0) {
                lw.nK[g] = K;
                lw.nKz[g] = Kz;
                lw.nrho[g] = rho;
                lw.ntol[g] = tol;
                lw.nzn[g] = S.nzn[j];
            }
        }

        // level diagnostics: one set of atomics per CTA and level
        if (x == 0) {
            brdc_level_diagnostics *dg = &a.w.hdr->diag[k];
            int skz = 0, sk = 0, kmax = 0;
            long long sk2 = 0;
            for (int q = 0; q < nk; ++q) {
                skz += S.nKz[q];
                sk += S.nK[q];
                kmax = max(kmax, S.nK[q]);
                sk2 += (long long)S.nK[q] * S.nK[q];
            }
            if (!A.ckpt) {
                atomicAdd(&dg->merge_count, nk);
                atomicAdd(&dg->size_sum, R);
                atomicAdd(&dg->dd_before_sum, skz);
                atomicAdd(&dg->dd_after_sum, sk);
                atomicMax(&dg->dd_after_max, kmax);
                atomicAdd((unsigned long long *)&dg->dd_after_sq_sum, (unsigned long long)sk2);
                dg->threads_per_root = 1;
            }
            if (S.it_sum != 0) {
                atomicAdd(&dg->secular_iter_sum, S.it_sum);
                atomicMax(&dg->secular_iter_max, S.it_max);
            }
            if (S.it_failed != 0) {
                atomicAdd(&dg->secular_iter_failed, S.it_failed);
                atomicAdd(&a.w.hdr->nonconv, S.it_failed);
            }
            S.it_sum = 0;
            S.it_max = 0;
            S.it_failed = 0;
        }

        // placement in ascending order (ties: roots, small-z, rotated)
        if (j >= 0) {
            const int q = x - s;
            const int ndz = m - Kz, ndg = Kz - K;
            const double *zdl = S.zd + s, *gdl = S.gd + s, *rl = S.rlam + s;
            double val, fo = 0.0, lo = 0.0;
            int pos;
            if (q < K) {
                val = rl[q];
                pos = q + lower_bound_d(zdl, ndz, val) + lower_bound_d(gdl, ndg, val);
                if (!top) {
                    fo = S.rf[s + q];
                    lo = S.rl[s + q];
                }
            } else if (q < K + ndz) {
                const int u = q - K;
                val = zdl[u];
                pos = u + upper_bound_d(rl, K, val) + lower_bound_d(gdl, ndg, val);
                fo = S.zf[s + u];
                lo = S.zl[s + u];
            } else {
                const int u = q - K - ndz;
                val = gdl[u];
                pos = u + upper_bound_d(rl, K, val) + upper_bound_d(zdl, ndz, val);
                fo = S.gf[s + u];
                lo = S.gl[s + u];
            }
            if (top) {
                a.W[gsub + s + pos] = val * wsc;
            } else {
                S.cd[s + pos] = val;
                S.cf[s + pos] = fo;
                S.cl[s + pos] = lo;
            }
        }
        __syncthreads();
    }

    // the subtree root's spectrum and rows for the per-level merges above
    if (!inst_top && x < R) {
        A.out_d[gsub + x] = S.cd[x];
        A.out_f[gsub + x] = S.cf[x];
        A.out_l[gsub + x] = S.cl[x];
    }
}

} // namespace brdc
