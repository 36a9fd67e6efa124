// brdc_level.cuh -- one merge level in one kernel.
//
// Above the subtree kernel the merges are few and large (a few thousand
// rows to the whole matrix), but for spectra that deflate heavily they
// leave only a few hundred poles each, and the per-level kernels spend a
// level on launches and global round trips -- short chains of dependent
// latencies.  k_level runs every step of a level for one merge node in a
// cluster of C CTAs (C = 1 allowed):
//   rank merge of the two children (a merge path through shared memory),
//   deflation (the phases of k_merge_deflate / k_merge_deflate_cl),
//   secular roots, Loewner weights and boundary rows of the K <= kLvlMaxK
//   poles in shared memory, the roots split over the cluster's CTAs and the
//   results gathered through distributed shared memory,
//   placement.
// Every rule is the per-level kernels' own (deflation tests, compaction
// order, rotations, the secular state machine, tie order of the placement),
// so deflation and placement decide exactly as they do; only the lanes that
// share a root's sweep differ, which moves the sums' rounding.  A node with
// more than kLvlMaxK poles stops after its deflation and is counted in the
// level's nbig; the last CTA then builds the level plan for exactly those
// nodes (big_k = kLvlMaxK), and k_sweeps finishes them (it returns at once
// when there are none).  Every write lands where the per-level kernels put
// it, so the workspace slices of a checkpointed solve serve the adjoint
// unchanged.
#pragma once

#include "brdc_kernels.cuh"

namespace brdc {

constexpr int kLvlThreads = 512;
constexpr int kLvlMaxK = 1024;       // poles a node takes through the roots in shared memory
constexpr int kLvlSamples = 4096;    // samples of a sorted list staged in shared memory
constexpr int kLvlRowsPerCta = 4096; // merge rows per CTA the launch aims at
constexpr int kLvlBatch = 4;         // rows a thread moves per pass (loads issued together)
constexpr int kLvlMergeChunk = 4096; // merged positions per chunk of the merge path
// Merges of at most this many rows are deflated by CTA 0 of their cluster
// alone (two chunks of 2048 rows at most), which measured faster than
// spreading them over the cluster with its count exchanges and barriers
// (uniform 65,536, level 7: 53 -> 48 us); 8192 gained nothing more, 16384
// lost.
constexpr int kLvlSoloDeflRows = 4096;

struct LvlSmem {
    double pd[kLvlMaxK], pz[kLvlMaxK], pf[kLvlMaxK], pl[kLvlMaxK], pw[kLvlMaxK];
    double rdo[kLvlMaxK], rtau[kLvlMaxK];
    double stage[2 * kLvlSamples];       // staged sorted lists of the placement
    double red[32];
    int iscan[32];
    double s_val;                        // cluster exchange
    int msplit[2];                       // merge-path splits of the current chunk
    int s_cnt;
    int s_kz;                            // CTA 0's deflation results for its peers
    double s_zn;                         // (s_val still holds max|z| for their reads)
    int s_rot;                           // this CTA rotated close poles out
    int s_last;
    uint64_t bar;                        // completion of the pole copies
};

// The merge uses pd .. stage as one scratch buffer (the poles are staged
// only after it), the placement pz .. stage (after the roots are gathered);
// the kernel addresses both from the raw shared-memory base.
static_assert(offsetof(LvlSmem, stage) == offsetof(LvlSmem, pd) + 7 * kLvlMaxK * sizeof(double),
              "pd .. rtau and stage must be contiguous");
static_assert(3 * kLvlMergeChunk <= 7 * kLvlMaxK + 2 * kLvlSamples,
              "the merge scratch must fit in pd .. stage");
static_assert(3 * kLvlMergeChunk <= 6 * kLvlMaxK + 2 * kLvlSamples,
              "the placement scratch must fit in pz .. stage");

// A sorted list in global memory with every Q-th element staged in shared
// memory.  A bound takes a binary search of the samples, then one scan of
// the (Q-1)-element window between two samples, so it is exact.
struct StagedList {
    const double *g; // the list
    const double *s; // s[i] = g[i Q]
    int n, Q, ns;
};

template <int T>
__device__ inline StagedList stage_list(double *dst, const double *g, int n) {
    StagedList L;
    L.g = g;
    L.s = dst;
    L.n = n;
    L.Q = n <= kLvlSamples ? 1 : (n + kLvlSamples - 1) / kLvlSamples;
    L.ns = (n + L.Q - 1) / L.Q;
    for (int i = threadIdx.x; i < L.ns; i += T) {
        dst[i] = g[(long long)i * L.Q];
    }
    return L;
}

// Step 1 of a bound: samples that pass (< v, or <= v for UPPER).
template <bool UPPER>
__device__ inline int staged_coarse(const StagedList &L, double v) {
    return UPPER ? upper_bound_d(L.s, L.ns, v) : lower_bound_d(L.s, L.ns, v);
}

// Step 2: elements that pass.  g[(c-1)Q] passes and g[cQ] (if any) fails,
// so only the window between them is read.
template <bool UPPER>
__device__ inline int staged_fine(const StagedList &L, int c, double v) {
    if (L.Q == 1 || c == 0) {
        return c * L.Q < L.n ? c * L.Q : L.n;
    }
    const int lo = (c - 1) * L.Q + 1;
    const int hi = c * L.Q < L.n ? c * L.Q : L.n;
    int cnt = lo;
    if (L.Q <= 8) {
        double t[7];
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            t[q] = lo + q < hi ? L.g[lo + q] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            cnt += (lo + q < hi) && (UPPER ? t[q] <= v : t[q] < v);
        }
        return cnt;
    }
    for (int j = lo; j < hi; ++j) {
        cnt += UPPER ? (L.g[j] <= v) : (L.g[j] < v);
    }
    return cnt;
}

// ---------------------------------------------------------------- merge
// The rank merge of a node's two sorted children as a merge path: CTA r of
// the cluster writes the merged positions [e0, e1), chunk by chunk.  For a
// chunk [oc, oe) the CTA finds how many left-child elements precede oc and
// oe (left wins ties: A[i] goes before B[j] iff A[i] <= B[j]), loads the two
// child ranges that fill the chunk into shared memory with coalesced loads,
// and every thread takes merged positions of the chunk by a binary search
// of the merge path in shared memory.  Each child element is read once and
// every store is coalesced; the order is exactly the rank merge's.

// Left-child elements among the first o merged elements, by a G-ary search
// of the merge path (G = T/2 threads, t = this thread's index in its half;
// the two halves of the CTA search for two positions at once).  Every
// thread of the CTA calls it; cnt points at 4 ints of shared memory.
template <int T>
__device__ inline int merge_split2(const double *A, int m1, const double *B, int m2, int o,
                                   int *cnt) {
    constexpr int G = T / 2;
    const int h = threadIdx.x / G, t = threadIdx.x % G;
    int lo = max(0, o - m2), hi = min(o, m1);
    if (threadIdx.x < 4) {
        cnt[threadIdx.x] = 0;
    }
    // invariant: the split (the smallest i with !(A[i] <= B[o-i-1])) lies in
    // [lo, hi]; at hi the test fails by definition
    for (int round = 0;; ++round) {
        if (!__syncthreads_or(lo < hi)) {
            break;
        }
        const int par = round & 1;
        if (threadIdx.x == 0) {
            cnt[(par ^ 1) * 2] = 0;
            cnt[(par ^ 1) * 2 + 1] = 0;
        }
        const int step = lo < hi ? (hi - lo + G - 1) / G : 1;
        const int c = lo + t * step;
        // c < hi <= min(o, m1), and c >= lo >= o - m2: both reads in range
        const bool good = lo < hi && c < hi && A[c] <= B[o - c - 1];
        const unsigned b = __ballot_sync(0xffffffffu, good);
        if ((threadIdx.x & 31) == 0 && b != 0u) {
            atomicAdd(&cnt[par * 2 + h], __popc(b));
        }
        __syncthreads();
        const int nt = cnt[par * 2 + h];
        if (lo < hi) {
            if (nt == 0) {
                hi = lo;
            } else {
                const int nlo = lo + (nt - 1) * step + 1;
                hi = min(hi, lo + nt * step);
                lo = nlo;
            }
        }
    }
    return lo;
}

// The merged lists md, mz, mf, ml, morig of positions [e0, e1) of node gs
// (left child rows [0, m1), right child [m1, m)); returns this thread's
// max |z|.  buf holds 3 * kLvlMergeChunk doubles of scratch; cnt 4 ints.
template <int T>
__device__ double level_merge(const Ws &w, long long gs, int m1, int m, int e0, int e1,
                              double *buf, int *cnt, int *split) {
    const int m2 = m - m1;
    const double *A = w.cd + gs, *B = w.cd + gs + m1;
    double *bd = buf, *bf = buf + kLvlMergeChunk, *bl = buf + 2 * kLvlMergeChunk;
    const int x = threadIdx.x;
    double lz = 0.0;
    for (int oc = e0; oc < e1; oc += kLvlMergeChunk) {
        const int oe = min(e1, oc + kLvlMergeChunk);
        const int s = merge_split2<T>(A, m1, B, m2, x < T / 2 ? oc : oe, cnt);
        if (x == 0) {
            split[0] = s;
        }
        if (x == T / 2) {
            split[1] = s;
        }
        __syncthreads();
        const int a0 = split[0], a1 = split[1];
        const int na = a1 - a0, n = oe - oc;
        const int b0 = oc - a0;
        // the two child ranges, left then right, into shared memory
        for (int u = x; u < n; u += T) {
            const long long src = u < na ? gs + a0 + u : gs + m1 + b0 + (u - na);
            bd[u] = w.cd[src];
            bf[u] = w.cf[src];
            bl[u] = w.cl[src];
        }
        __syncthreads();
        const int nb = n - na;
        for (int k = x; k < n; k += T) {
            int lo = max(0, k - nb), hi = min(k, na);
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (bd[mid] <= bd[na + k - mid - 1]) {
                    lo = mid + 1;
                } else {
                    hi = mid;
                }
            }
            const int i = lo, j = k - lo;
            const bool left = i < na && (j >= nb || bd[i] <= bd[na + j]);
            const int u = left ? i : na + j;
            const double r = left ? bl[u] : bf[u];
            const double z = r / kSqrt2;
            const long long o = gs + oc + k;
            w.md[o] = bd[u];
            w.mz[o] = z;
            w.mf[o] = left ? bf[u] : 0.0;
            w.ml[o] = left ? 0.0 : bl[u];
            w.morig[o] = left ? a0 + i : m1 + b0 + j;
            lz = fmax(lz, fabs(z));
        }
        __syncthreads();
    }
    return lz;
}

// Placement of a node none of whose poles was rotated out: its ascending
// order is the merge of the roots (R, in shared memory) and the small-z
// list (zd, zf, zl), roots first on ties -- the order the three-list rank
// rule gives -- taken as a merge path like the rank merge: chunk splits by
// merge_split2, the small-z range loaded coalesced into shared memory
// (buf: pz .. stage, free once the roots are gathered), every output
// stored coalesced.  Outputs [e0, e1) of the node; at an instance root the
// values go to W.
template <int T>
__device__ void level_place_merge(const KArgs &a, const Ws &w, LvlSmem &S, double *buf,
                                  long long gs, long long po, int K, int ndz, int e0, int e1,
                                  bool top, double wsc) {
    const double *R = S.pd;
    const double *Z = w.zd + gs;
    double *zd = buf, *zf = buf + kLvlMergeChunk, *zl = buf + 2 * kLvlMergeChunk;
    const int x = threadIdx.x;
    for (int oc = e0; oc < e1; oc += kLvlMergeChunk) {
        const int oe = min(e1, oc + kLvlMergeChunk);
        const int sp = merge_split2<T>(R, K, Z, ndz, x < T / 2 ? oc : oe, S.iscan);
        if (x == 0) {
            S.msplit[0] = sp;
        }
        if (x == T / 2) {
            S.msplit[1] = sp;
        }
        __syncthreads();
        const int r0 = S.msplit[0], r1 = S.msplit[1];
        const int nr = r1 - r0, n = oe - oc, nz = n - nr;
        const int z0 = oc - r0;
        for (int u = x; u < nz; u += T) {
            const long long src = gs + z0 + u;
            zd[u] = w.zd[src];
            zf[u] = w.zf[src];
            zl[u] = w.zl[src];
        }
        __syncthreads();
        for (int k = x; k < n; k += T) {
            int lo = max(0, k - nz), hi = min(k, nr);
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (R[r0 + mid] <= zd[k - mid - 1]) {
                    lo = mid + 1;
                } else {
                    hi = mid;
                }
            }
            const int i = lo, j = k - lo;
            const bool root = i < nr && (j >= nz || R[r0 + i] <= zd[j]);
            const long long o = gs + oc + k;
            const double val = root ? R[r0 + i] : zd[j];
            if (top) {
                a.W[o] = val * wsc;
            } else {
                w.nd[o] = val;
                w.nf[o] = root ? __ldcg(w.rf + po + r0 + i) : zf[j];
                w.nl[o] = root ? __ldcg(w.rl + po + r0 + i) : zl[j];
            }
        }
        __syncthreads();
    }
}

// Roots, Loewner weights and boundary rows of one node with 1 <= K <=
// kLvlMaxK poles, by all C CTAs of its cluster: CTA r takes the roots (and
// poles) [r P, (r+1) P), P = ceil(K / C), and gathers the others' from their
// shared memory.  Results go to the workspace where k_secular, k_lowner and
// k_rows put them; on return every CTA holds all rdo/rtau.  The caller ends
// with a cluster barrier, after which no CTA reads a peer's shared memory.
template <int T>
__device__ void level_roots(LvlSmem &S, cooperative_groups::cluster_group &cl, const KArgs &a,
                            const NodeGeom &G, int K, double rho, double zn, int C, int rank) {
    const Ws &w = a.w;
    const long long po = G.poff;
    const int x = threadIdx.x, lane = x & 31;
    const double eps = DBL_EPSILON;
    const int max_iter = a.w.hdr->max_iter;
    // The node's poles, weights and rows into shared memory by four bulk
    // copies (cp.async.bulk, one thread issues them) completing on one
    // mbarrier.  The pole slice starts 16-byte aligned; an odd K copies one
    // element more, which the padded slice holds.  The cluster's deflation
    // wrote these arrays with ordinary stores just before (released by the
    // cluster barrier), hence the proxy fence before the copies.  A wait
    // past the handle's limit is followed by a bounded drain, so the block
    // never moves on with copies in flight; only a failed drain records an
    // error.
    {
        const unsigned bytes = (unsigned)(((K + 1) & ~1) * sizeof(double));
        if (x == 0) {
            mbar_init(&S.bar, 1);
            fence_mbar_init();
            fence_proxy_async_global();
            mbar_expect_tx(&S.bar, 4u * bytes);
            bulk_g2s(S.pd, w.pd + po, bytes, &S.bar);
            bulk_g2s(S.pz, w.pz + po, bytes, &S.bar);
            bulk_g2s(S.pf, w.pf + po, bytes, &S.bar);
            bulk_g2s(S.pl, w.pl + po, bytes, &S.bar);
        }
        __syncthreads();
        if (!mbar_wait(&S.bar, 0u, w.hdr->wait_ns) && !mbar_wait(&S.bar, 0u, kDrainWaitNs)) {
            record_error(w.hdr, kErrBarrierTimeout);
        }
        __syncthreads();
    }
    const int P = (K + C - 1) / C;
    const int r0 = min(K, rank * P), r1 = min(K, r0 + P);
    if (K == 1) {
        if (rank == 0 && x == 0) {
            const double t = rho * S.pz[0] * S.pz[0];
            S.rdo[0] = S.pd[0];
            S.rtau[0] = t;
            w.rorg[po] = 0;
            w.rdo[po] = S.pd[0];
            w.rtau[po] = t;
            w.rlam[po] = S.pd[0] + t;
        }
    } else if (r1 > r0) {
        // tp lanes per root (the largest power of two that covers the CTA's
        // roots in one pass), each group iterating its root to convergence:
        // no barrier between sweeps
        const int nmine = r1 - r0;
        int tp = 1;
        while (tp < 32 && nmine * tp * 2 <= T) {
            tp <<= 1;
        }
        const int per = T / tp, l2 = x & (tp - 1);
        int its = 0, itm = 0, itf = 0;
        for (int base = 0; base < nmine; base += per) {
            const int r = r0 + base + x / tp;
            const bool act = r < r1;
            SecRoot st;
            if (act) {
                sec_init(st, r, K, S.pd, S.pz, rho, zn);
            } else {
                st.stage = 2;
            }
            const int pmin = r < K - 2 ? r : K - 2;
            for (;;) {
                SecSums sum;
                sec_zero(sum);
                const bool live = act && st.stage != 2;
                if (live) {
                    secular_span(sum, st, 0, K, l2, tp, pmin, r + 1,
                                 [&](int u, double *du, double *zu) {
                                     *du = S.pd[u];
                                     *zu = S.pz[u];
                                 });
                }
                sums_reduce(sum, tp);
                if (live) {
                    sec_after_sweep(st, sum, eps, max_iter);
                }
                if (__all_sync(kFull, !act || st.stage == 2)) {
                    break;
                }
            }
            if (act && l2 == 0) {
                S.rdo[r] = st.dorg;
                S.rtau[r] = st.tau;
                w.rorg[po + r] = st.org;
                w.rdo[po + r] = st.dorg;
                w.rtau[po + r] = st.tau;
                w.rlam[po + r] = st.dorg + st.tau;
                its += st.iter;
                itm = max(itm, st.iter);
                itf += st.failed;
            }
        }
        // iteration counters, one warp at a time
        its = __reduce_add_sync(kFull, its);
        itm = __reduce_max_sync(kFull, itm);
        itf = __reduce_add_sync(kFull, itf);
        if (lane == 0 && its != 0) {
            brdc_level_diagnostics *dg = &w.hdr->diag[a.k];
            atomicAdd(&dg->secular_iter_sum, its);
            atomicMax(&dg->secular_iter_max, itm);
            if (itf != 0) {
                atomicAdd(&dg->secular_iter_failed, itf);
                atomicAdd(&w.hdr->nonconv, itf);
            }
        }
    }
    // every CTA: the other CTAs' roots
    cl.sync();
    for (int i = x; i < K; i += T) {
        const int owner = i / P;
        if (owner != rank) {
            S.rdo[i] = *cl.map_shared_rank(&S.rdo[i], owner);
            S.rtau[i] = *cl.map_shared_rank(&S.rtau[i], owner);
        }
    }
    __syncthreads();
    if (G.depth == 0) {
        return; // an instance root: no parent reads its rows
    }

    // Loewner weights (sqrt(rho) z) of this CTA's poles, tpr lanes per pole
    const int nmine = r1 - r0;
    int tpr = 1;
    while (tpr < 32 && nmine * tpr * 2 <= T) {
        tpr <<= 1;
    }
    const int per = T / tpr, gl = x & (tpr - 1);
    for (int base = 0; base < nmine; base += per) {
        const int i = r0 + base + x / tpr;
        double prod = 1.0;
        if (i < r1) {
            const double di = S.pd[i];
            int q = gl;
            for (; q + tpr < K; q += 2 * tpr) {
                const int q2 = q + tpr;
                const double dl = (di - S.rdo[q]) - S.rtau[q];
                const double dl2 = (di - S.rdo[q2]) - S.rtau[q2];
                prod *= lowner_pair(dl, q == i ? 1.0 : di - S.pd[q], dl2,
                                    q2 == i ? 1.0 : di - S.pd[q2]);
            }
            if (q < K) {
                const double dl = (di - S.rdo[q]) - S.rtau[q];
                prod *= dl * brdc_rcp(q == i ? 1.0 : di - S.pd[q]);
            }
        }
        prod = group_prod(prod, tpr);
        if (i < r1 && gl == 0) {
            const double zi = S.pz[i];
            const double mag = sqrt(fmax(-prod, 0.0));
            double wi = zi < 0.0 ? -mag : mag;
            if (!(mag > 0.0) || !isfinite(mag)) {
                wi = zi * sqrt(rho);
            }
            S.pw[i] = wi;
            w.pw[po + i] = wi;
        }
    }
    cl.sync();
    for (int i = x; i < K; i += T) {
        const int owner = i / P;
        if (owner != rank) {
            S.pw[i] = *cl.map_shared_rank(&S.pw[i], owner);
        }
    }
    __syncthreads();

    // boundary rows of this CTA's roots, tpr lanes per root
    for (int base = 0; base < nmine; base += per) {
        const int r = r0 + base + x / tpr;
        double a1 = 0.0, a2 = 0.0, s2 = 0.0;
        if (r < r1) {
            const double dorg = S.rdo[r], tau = S.rtau[r];
            int i = gl;
            for (; i + tpr < K; i += 2 * tpr) {
                const int i2 = i + tpr;
                double u, u2;
                row_pair(S.pw[i], (S.pd[i] - dorg) - tau, S.pw[i2], (S.pd[i2] - dorg) - tau, &u,
                         &u2);
                s2 += u * u;
                a1 += S.pf[i] * u;
                a2 += S.pl[i] * u;
                s2 += u2 * u2;
                a1 += S.pf[i2] * u2;
                a2 += S.pl[i2] * u2;
            }
            if (i < K) {
                const double dl = (S.pd[i] - dorg) - tau;
                const double u = (dl != 0.0) ? S.pw[i] * brdc_rcp(dl) : 0.0;
                s2 += u * u;
                a1 += S.pf[i] * u;
                a2 += S.pl[i] * u;
            }
        }
        s2 = group_sum(s2, tpr);
        a1 = group_sum(a1, tpr);
        a2 = group_sum(a2, tpr);
        if (r < r1 && gl == 0) {
            const double nrm = sqrt(s2);
            w.rf[po + r] = nrm > 0.0 ? a1 / nrm : 0.0;
            w.rl[po + r] = nrm > 0.0 ? a2 / nrm : 0.0;
        }
    }
}

// The level plan for the merges k_level leaves to k_sweeps: taken by the
// last CTA of the launch (every node's scalars are written before its CTAs
// take their tickets), and only when there are such merges.
template <int T>
__device__ void level_ticket(const KArgs &a, LvlSmem &S) {
    if (!a.plan_inline) {
        return; // k_plan runs after the launch
    }
    LevelCtl *c = &a.w.hdr->lvl[a.k];
    if (threadIdx.x == 0) {
        __threadfence();
        const int t = atomicAdd(&c->ticket, 1);
        S.s_last = (t == (int)gridDim.x - 1) && (atomicAdd(&c->nbig, 0) > 0);
    }
    __syncthreads();
    if (S.s_last) {
        __threadfence();
        level_plan<T>(a, S.red, S.iscan);
    }
}

// One merge level, a cluster of C CTAs per node.  CTA r of the cluster
// merges and places the rows [r SE, (r+1) SE) and deflates its share as
// k_merge_deflate_cl does.
template <int T>
__global__ void __launch_bounds__(T, 1) k_level(KArgs a) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    namespace cg = cooperative_groups;
    extern __shared__ __align__(16) unsigned char lvl_raw[];
    LvlSmem &S = *reinterpret_cast<LvlSmem *>(lvl_raw);
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks();
    const int rank = (int)cl.block_rank();
    const int g = blockIdx.x / C;
    const NodeGeom G = node_geom(a.F, a.k, g);
    const Ws &w = a.w;
    const long long gs = G.gstart;
    const int m = G.m, m1 = G.m1;
    const int x = threadIdx.x;
    constexpr int chunk = kDeflEPT * T;
    constexpr int B = kLvlBatch;
    double rho, maxd;
    defl_node_scalars(a, G, &rho, &maxd);

    // ------------------------------------------------ rank merge
    // (left wins ties), as k_merge, by the merge path; max|z| on the way
    const int SE = (m + C - 1) / C;
    const int e0 = min(m, rank * SE), e1 = min(m, e0 + SE);
    double lz = level_merge<T>(w, gs, m1, m, e0, e1,
                               reinterpret_cast<double *>(lvl_raw + offsetof(LvlSmem, pd)),
                               S.iscan, S.msplit);
    lz = block_max<T>(lz, S.red);
    if (x == 0) {
        S.s_val = lz;
    }
    // the cluster barrier releases and acquires at cluster scope, which
    // orders the global writes of every phase for the peer CTAs
    cl.sync();
    double maxz = 0.0;
    for (int r = 0; r < C; ++r) {
        maxz = fmax(maxz, *cl.map_shared_rank(&S.s_val, r));
    }
    const double tol = kDeflTolScale * DBL_EPSILON * fmax(maxd, maxz);

    // ------------------------------------------------ deflation
    int K, Kz;
    double zn;
    if (C == 1) {
        Kz = defl_compact_active<T>(w, gs, 0, m, rho, tol, 0, 0, S.iscan);
        __syncthreads();
        defl_close_walk<T>(w, gs, Kz, tol, 0, Kz);
        __syncthreads();
        zn = defl_compact_poles<T>(w, gs, G.poff, 0, Kz, 0, 0, S.iscan, &K);
        zn = block_sum<T>(zn, S.red);
    } else if (m <= kLvlSoloDeflRows || m <= ((m + C - 1) / C + chunk - 1) / chunk * chunk) {
        // a small merge (or one that lies in CTA 0's deflation slice alone,
        // the slices being whole chunks): CTA 0 deflates it as one CTA per
        // node does, with no counts to exchange, and its peers wait at one
        // cluster barrier
        if (rank == 0) {
            Kz = defl_compact_active<T>(w, gs, 0, m, rho, tol, 0, 0, S.iscan);
            __syncthreads();
            defl_close_walk<T>(w, gs, Kz, tol, 0, Kz);
            __syncthreads();
            zn = defl_compact_poles<T>(w, gs, G.poff, 0, Kz, 0, 0, S.iscan, &K);
            zn = block_sum<T>(zn, S.red);
            if (x == 0) {
                S.s_cnt = K;
                S.s_kz = Kz;
                S.s_zn = zn;
            }
        }
        cl.sync();
        K = *cl.map_shared_rank(&S.s_cnt, 0);
        Kz = *cl.map_shared_rank(&S.s_kz, 0);
        zn = *cl.map_shared_rank(&S.s_zn, 0);
    } else {
        const int SD = ((m + C - 1) / C + chunk - 1) / chunk * chunk;
        const int r0 = min(m, rank * SD), r1 = min(m, r0 + SD);
        const int na = defl_count_active<T>(w, gs, r0, r1, rho, tol, S.iscan);
        if (x == 0) {
            S.s_cnt = na;
        }
        cl.sync();
        int off_a = 0;
        Kz = 0;
        for (int r = 0; r < C; ++r) {
            const int cn = *cl.map_shared_rank(&S.s_cnt, r);
            off_a += r < rank ? cn : 0;
            Kz += cn;
        }
        defl_compact_active<T>(w, gs, r0, r1, rho, tol, off_a, r0 - off_a, S.iscan);
        cl.sync();
        const int A = (Kz + C - 1) / C;
        const int rot = __syncthreads_or(
            defl_close_walk<T>(w, gs, Kz, tol, min(Kz, rank * A), min(Kz, rank * A + A)));
        if (x == 0) {
            S.s_rot = rot;
        }
        cl.sync();
        bool any_rot = false;
        for (int r = 0; r < C; ++r) {
            any_rot |= *cl.map_shared_rank(&S.s_rot, r) != 0;
        }
        const int S2 = ((Kz + C - 1) / C + chunk - 1) / chunk * chunk;
        const int q0 = min(Kz, rank * S2), q1 = min(Kz, q0 + S2);
        int off_p = q0;
        K = Kz;
        if (any_rot) {
            // some entries were rotated out: count the poles of every
            // slice (with none, every active entry is a pole)
            const int np = defl_count_poles<T>(w, gs, q0, q1, S.iscan);
            if (x == 0) {
                S.s_cnt = np;
            }
            cl.sync();
            off_p = 0;
            K = 0;
            for (int r = 0; r < C; ++r) {
                const int cn = *cl.map_shared_rank(&S.s_cnt, r);
                off_p += r < rank ? cn : 0;
                K += cn;
            }
        }
        int end_p;
        double zp = defl_compact_poles<T>(w, gs, G.poff, q0, q1, off_p, q0 - off_p, S.iscan,
                                          &end_p);
        zp = block_sum<T>(zp, S.red);
        if (x == 0) {
            S.s_val = zp;
        }
        cl.sync();
        zn = 0.0;
        for (int r = 0; r < C; ++r) {
            zn += *cl.map_shared_rank(&S.s_val, r);
        }
    }
    if (rank == 0 && x == 0) {
        w.nK[g] = K;
        w.nKz[g] = Kz;
        w.nrho[g] = rho;
        w.ntol[g] = tol;
        w.nzn[g] = zn;
        // level counters of the reference's diagnostics, one node at a time
        brdc_level_diagnostics *dg = &w.hdr->diag[a.k];
        atomicAdd(&dg->merge_count, 1);
        atomicAdd(&dg->size_sum, m);
        atomicAdd(&dg->dd_before_sum, Kz);
        atomicAdd(&dg->dd_after_sum, K);
        atomicMax(&dg->dd_after_max, K);
        atomicAdd((unsigned long long *)&dg->dd_after_sq_sum,
                  (unsigned long long)K * (unsigned long long)K);
        if (K > kLvlMaxK) {
            atomicAdd(&w.hdr->lvl[a.k].nbig, 1);
        }
    }
    if (K > kLvlMaxK) {
        // no CTA leaves while a peer may still read its shared memory
        cl.sync();
        level_ticket<T>(a, S);
        return; // k_sweeps finishes this node
    }

    // ------------------------------------------------ roots
    if (K > 0) {
        level_roots<T>(S, cl, a, G, K, rho, zn, C, rank);
    }
    cl.sync();

    // ------------------------------------------------ placement
    // ascending order, ties: roots, small-z deflated, rotated out (as
    // place_rows)
    const int ndz = m - Kz, ndg = Kz - K;
    const long long po = G.poff;
    for (int i = x; i < K; i += T) {
        S.pd[i] = S.rdo[i] + S.rtau[i]; // = rlam, bit for bit
    }
    const bool top = (G.depth == 0);
    const double wsc = inst_unscale(w, G.inst);
    if (ndg == 0) {
        __syncthreads();
        level_place_merge<T>(a, w, S, reinterpret_cast<double *>(lvl_raw + offsetof(LvlSmem, pz)),
                             gs, po, K, ndz, e0, e1, top, wsc);
    } else {
        const StagedList LZ = stage_list<T>(S.stage, w.zd + gs, ndz);
        const StagedList LG = stage_list<T>(S.stage + kLvlSamples, w.gd + gs, ndg);
        __syncthreads();
        for (int s0 = e0 + x; s0 < e1; s0 += B * T) {
            double val[B], fo[B], lo[B];
            int pos[B];
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const int s = s0 + u * T < e1 ? s0 + u * T : s0;
                if (s < K) {
                    val[u] = S.pd[s];
                    fo[u] = top ? 0.0 : __ldcg(w.rf + po + s);
                    lo[u] = top ? 0.0 : __ldcg(w.rl + po + s);
                } else if (s < K + ndz) {
                    val[u] = w.zd[gs + s - K];
                    fo[u] = w.zf[gs + s - K];
                    lo[u] = w.zl[gs + s - K];
                } else {
                    val[u] = w.gd[gs + s - K - ndz];
                    fo[u] = w.gf[gs + s - K - ndz];
                    lo[u] = w.gl[gs + s - K - ndz];
                }
            }
            // each row searches the two lists it is not in (rows of one warp
            // are consecutive, so the branches split few warps)
            int cz[B], cgr[B];
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const int s = s0 + u * T;
                cz[u] = 0;
                cgr[u] = 0;
                if (s < K) {
                    cz[u] = staged_coarse<false>(LZ, val[u]);
                    cgr[u] = staged_coarse<false>(LG, val[u]);
                } else if (s < K + ndz) {
                    cgr[u] = staged_coarse<false>(LG, val[u]);
                } else {
                    cz[u] = staged_coarse<true>(LZ, val[u]); // rotated out: ties after small-z
                }
            }
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const int s = s0 + u * T;
                if (s < K) {
                    pos[u] = s + staged_fine<false>(LZ, cz[u], val[u]) +
                             staged_fine<false>(LG, cgr[u], val[u]);
                } else if (s < K + ndz) {
                    pos[u] = (s - K) + upper_bound_d(S.pd, K, val[u]) +
                             staged_fine<false>(LG, cgr[u], val[u]);
                } else {
                    pos[u] = (s - K - ndz) + upper_bound_d(S.pd, K, val[u]) +
                             staged_fine<true>(LZ, cz[u], val[u]);
                }
            }
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const int s = s0 + u * T;
                if (s < e1) {
                    const long long o = gs + pos[u];
                    if (top) {
                        a.W[o] = val[u] * wsc;
                    } else {
                        w.nd[o] = val[u];
                        w.nf[o] = fo[u];
                        w.nl[o] = lo[u];
                    }
                }
            }
        }
    }
    level_ticket<T>(a, S);
}

} // namespace brdc
