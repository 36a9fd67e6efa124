// brdc_kernels.cuh -- sm_100a kernels of the forward BR solve.
//
// One forest level runs four kernels:
//   k_merge_deflate  one CTA per merge: z from the children's boundary rows,
//                    merge of the two sorted child spectra, small-z and
//                    close-pole deflation with Givens rotations of z and of
//                    both boundary rows, compaction, work plan of the level
//   k_secular        secular roots, TPR lanes per root, pole tiles staged in
//                    shared memory by cp.async.bulk
//   k_lowner         Loewner / Gu-Eisenstat recomputation of z
//   k_rows_place     first/last rows of the merged eigenvector matrix for
//                    every root, and the final sorted placement of all
//                    eigenvalues of the node
// The leaves are solved first by k_leaf (one warp per leaf, parallel
// cyclic Jacobi).
#pragma once

#include <cfloat>
#include <cstdint>

#include "brdc_common.cuh"
#include "brdc_secular.cuh"

namespace brdc {

struct KArgs {
    Forest F;
    Ws w;
    const double *D;
    const double *E;
    double *W;          // final eigenvalues
    int k;              // forest level
    int nodes;          // merges at this level
};

// ------------------------------------------------------------------ leaves
// One warp per leaf of <= 16 rows.  The leaf matrix (with the rank-one cut
// corrections D -= |E_cut| at both ends, gpu/src/tridiag_solver_extract.cuh:
// 104-117) is diagonalised by cyclic Jacobi with the round-robin ordering:
// 8 disjoint rotations per round, 15 rounds per sweep, applied by all 32
// lanes at once.  The reference runs a serial Jacobi on one thread per leaf
// (gpu/src/tridiag_solver_leaf.cuh:56-123).  Output: ascending eigenvalues,
// and the first and last rows of the eigenvector matrix in that order.
constexpr int kLeafWarps = 4;
constexpr int kLeafLd = 17;

__global__ void __launch_bounds__(kLeafWarps * 32)
    k_leaf(KArgs a, long long total_leaves) {
    __shared__ double sA[kLeafWarps][16 * kLeafLd];
    __shared__ double sV[kLeafWarps][16 * kLeafLd];
    __shared__ int sPart[kLeafWarps][16];
    __shared__ double sC[kLeafWarps][16];
    __shared__ double sS[kLeafWarps][16];
    __shared__ double sDiag[kLeafWarps][16];
    __shared__ int sRot[kLeafWarps][16];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *A = sA[warp];
    double *V = sV[warp];
    const double eps = DBL_EPSILON;
    int sweeps_max = 0;

    for (long long leaf = (long long)blockIdx.x * kLeafWarps + warp;
         leaf < total_leaves; leaf += (long long)gridDim.x * kLeafWarps) {
        const LeafGeom G = leaf_geom(a.F, leaf);
        const int s = G.s;
        for (int e = lane; e < 256; e += 32) {
            const int r = e >> 4, c = e & 15;
            A[r * kLeafLd + c] = 0.0;
            V[r * kLeafLd + c] = (r == c) ? 1.0 : 0.0;
        }
        __syncwarp();
        double amax = 0.0;
        if (lane < s) {
            double dv = a.D[G.gstart + lane];
            if (lane == 0 && G.gstart > G.istart) {
                dv -= fabs(a.E[G.gstart - 1]);
            }
            if (lane == s - 1 && G.gstart + s < G.iend) {
                dv -= fabs(a.E[G.gstart + s - 1]);
            }
            A[lane * kLeafLd + lane] = dv;
            amax = fabs(dv);
            if (lane + 1 < s) {
                const double ev = fabs(a.E[G.gstart + lane]);
                A[lane * kLeafLd + lane + 1] = ev;
                A[(lane + 1) * kLeafLd + lane] = ev;
                amax = fmax(amax, ev);
            }
        }
        amax = warp_max(amax);
        __syncwarp();
        const double thresh = 1.0e-3 * eps * amax;

        int sweep = 0;
        for (; sweep < 40; ++sweep) {
            double off = 0.0;
            for (int e = lane; e < 256; e += 32) {
                const int r = e >> 4, c = e & 15;
                if (r != c) {
                    off = fmax(off, fabs(A[r * kLeafLd + c]));
                }
            }
            off = warp_max(off);
            if (!(off > thresh)) {
                break;
            }
            for (int round = 0; round < 15; ++round) {
                if (lane < 8) {
                    int pa, pb;
                    if (lane == 0) {
                        pa = round;
                        pb = 15;
                    } else {
                        pa = (round + lane) % 15;
                        pb = (round + 15 - lane) % 15;
                    }
                    const int p = pa < pb ? pa : pb;
                    const int q = pa < pb ? pb : pa;
                    const double apq = A[p * kLeafLd + q];
                    const double app = A[p * kLeafLd + p];
                    const double aqq = A[q * kLeafLd + q];
                    double c = 1.0, sn = 0.0, t = 0.0;
                    int rot = 0;
                    if (fabs(apq) > thresh) {
                        const double theta = (aqq - app) / (2.0 * apq);
                        if (fabs(theta) > 1.0e150) {
                            t = 0.5 / theta;
                        } else {
                            t = (theta >= 0.0 ? 1.0 : -1.0) /
                                (fabs(theta) + sqrt(theta * theta + 1.0));
                        }
                        c = 1.0 / sqrt(t * t + 1.0);
                        sn = t * c;
                        rot = 1;
                    }
                    sPart[warp][p] = q;
                    sPart[warp][q] = p;
                    sC[warp][p] = c;
                    sC[warp][q] = c;
                    sS[warp][p] = -sn; // J(q,p)
                    sS[warp][q] = sn;  // J(p,q)
                    sRot[warp][p] = rot;
                    sRot[warp][q] = rot;
                    sDiag[warp][p] = app - t * apq;
                    sDiag[warp][q] = aqq + t * apq;
                }
                __syncwarp();
                double na[8], nv[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int e = lane + 32 * u;
                    const int r = e >> 4, c = e & 15;
                    const int rb = sPart[warp][r], cb = sPart[warp][c];
                    const double cr = sC[warp][r], sr = sS[warp][r];
                    const double cc = sC[warp][c], sc = sS[warp][c];
                    double v;
                    if (r == c) {
                        v = sRot[warp][r] ? sDiag[warp][r] : A[r * kLeafLd + r];
                    } else if (c == rb) {
                        v = sRot[warp][r] ? 0.0 : A[r * kLeafLd + c];
                    } else {
                        v = cr * (A[r * kLeafLd + c] * cc + A[r * kLeafLd + cb] * sc) +
                            sr * (A[rb * kLeafLd + c] * cc + A[rb * kLeafLd + cb] * sc);
                    }
                    na[u] = v;
                    nv[u] = V[r * kLeafLd + c] * cc + V[r * kLeafLd + cb] * sc;
                }
                __syncwarp();
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int e = lane + 32 * u;
                    const int r = e >> 4, c = e & 15;
                    A[r * kLeafLd + c] = na[u];
                    V[r * kLeafLd + c] = nv[u];
                }
                __syncwarp();
            }
        }
        sweeps_max = sweeps_max > sweep ? sweeps_max : sweep;

        // bitonic sort of (eigenvalue, column) over the 32 lanes
        double key = (lane < s) ? A[lane * kLeafLd + lane] : INFINITY;
        int col = lane;
        for (int size = 2; size <= 32; size <<= 1) {
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                const double ok = __shfl_xor_sync(0xffffffffu, key, stride);
                const int oc = __shfl_xor_sync(0xffffffffu, col, stride);
                const bool up = ((lane & size) == 0);
                const bool lower = ((lane & stride) == 0);
                const bool take_min = (up == lower);
                const bool swap = take_min ? (ok < key || (ok == key && oc < col))
                                           : (ok > key || (ok == key && oc > col));
                if (swap) {
                    key = ok;
                    col = oc;
                }
            }
        }
        if (lane < s) {
            const long long o = G.gstart + lane;
            if (G.top) {
                a.W[o] = key;
            } else {
                a.w.cd[o] = key;
                a.w.cf[o] = V[0 * kLeafLd + col];
                a.w.cl[o] = V[(s - 1) * kLeafLd + col];
            }
        }
        __syncwarp();
    }
    if (lane == 0 && sweeps_max > 0) {
        atomicMax(&a.w.hdr->leaf_sweeps_max, sweeps_max);
    }
}

// ------------------------------------------------------ merge + deflation
// One CTA per merge node.  Semantics of the reference GPU deflation
// (gpu/src/tridiag_solver_merge_kernels.cuh:1040-1102, 143-290, 326-439):
//   z = (last rows of the left child, first rows of the right child)/sqrt2,
//   rho = 2|E_cut|, tol = 8*eps*max(max|d|, max|z|), a pole stays active
//   when |rho*z| > tol; active poles are sorted ascending; runs of active
//   poles with gaps <= tol form clusters greedily (a new cluster starts when
//   a pole is more than tol above the cluster base); every member is rotated
//   into its base by lartg and deflated with its own d.
// The rotation is applied to both boundary rows with the same orientation
// as to z (new_b = c*b + s*t, new_t = -s*b + c*t), so the parent rows stay
// consistent with the rotated z.
template <int T>
__global__ void __launch_bounds__(T) k_merge_deflate(KArgs a) {
    __shared__ double red[32];
    __shared__ int iscan[32];
    __shared__ int s_last;
    const int g = blockIdx.x;
    const NodeGeom G = node_geom(a.F, a.k, g);
    const Ws &w = a.w;
    const long long gs = G.gstart;
    const int m = G.m, m1 = G.m1, m2 = G.m - G.m1;
    const double eps = DBL_EPSILON;
    const double isq2 = 0.70710678118654752440;

    const double *Ad = w.cd + gs;
    const double *Bd = w.cd + gs + m1;
    const double rho = 2.0 * fabs(a.E[gs + m1 - 1]);
    double maxd = fmax(fmax(fabs(Ad[0]), fabs(Ad[m1 - 1])),
                       fmax(fabs(Bd[0]), fabs(Bd[m2 - 1])));
    double lz = 0.0;
    for (int e = threadIdx.x; e < m; e += T) {
        const double z = (e < m1) ? w.cl[gs + e] * isq2 : w.cf[gs + e] * isq2;
        lz = fmax(lz, fabs(z));
    }
    const double maxz = block_max<T>(lz, red);
    const double tol = kDeflTolScale * eps * fmax(maxd, maxz);

    // merge of the two sorted child lists by rank in the sibling
    for (int e = threadIdx.x; e < m; e += T) {
        double x, z, f, l;
        int pos;
        if (e < m1) {
            x = Ad[e];
            pos = e + lower_bound_d(Bd, m2, x);
            z = w.cl[gs + e] * isq2;
            f = w.cf[gs + e];
            l = 0.0;
        } else {
            const int j = e - m1;
            x = Bd[j];
            pos = j + upper_bound_d(Ad, m1, x);
            z = w.cf[gs + e] * isq2;
            f = 0.0;
            l = w.cl[gs + e];
        }
        const long long o = gs + pos;
        w.md[o] = x;
        w.mz[o] = z;
        w.mf[o] = f;
        w.ml[o] = l;
        w.mflag[o] = fabs(rho * z) > tol ? 1 : 0;
        w.morig[o] = e;
    }
    __syncthreads();

    // compaction 1: small-z survivors (sorted) and small-z deflated (sorted)
    int carry_a = 0, carry_z = 0;
    for (int base = 0; base < m; base += 4 * T) {
        int fl[4];
        int cnt = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int idx = base + 4 * threadIdx.x + q;
            fl[q] = (idx < m) ? w.mflag[gs + idx] : 0;
            cnt += fl[q];
        }
        int tot;
        const int ex = block_exscan<T>(cnt, iscan, &tot);
        int ra = carry_a + ex;
        int rz = carry_z + (4 * threadIdx.x - ex);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int idx = base + 4 * threadIdx.x + q;
            if (idx < m) {
                const long long src = gs + idx;
                if (fl[q]) {
                    const long long o = gs + ra;
                    w.ad[o] = w.md[src];
                    w.az[o] = w.mz[src];
                    w.af[o] = w.mf[src];
                    w.al[o] = w.ml[src];
                    w.amap[o] = idx;
                    w.gmark[o] = 0;
                    ++ra;
                } else {
                    const long long o = gs + rz;
                    w.zd[o] = w.md[src];
                    w.zf[o] = w.mf[src];
                    w.zl[o] = w.ml[src];
                    ++rz;
                }
            }
        }
        const int valid = (m - base) < 4 * T ? (m - base) : 4 * T;
        carry_a += tot;
        carry_z += valid - tot;
    }
    const int Kz = carry_a;
    __syncthreads();

    // close-pole clusters: one thread walks each run of gaps <= tol
    for (int i = threadIdx.x; i < Kz; i += T) {
        const double di = w.ad[gs + i];
        const bool nxt = (i + 1 < Kz) && (w.ad[gs + i + 1] - di <= tol);
        const bool prv = (i > 0) && (di - w.ad[gs + i - 1] <= tol);
        if (!nxt || prv) {
            continue;
        }
        int base = i;
        double dbase = di;
        double zb = w.az[gs + i], fb = w.af[gs + i], lb = w.al[gs + i];
        int x = i + 1;
        double dprev = di;
        while (x < Kz) {
            const double dx = w.ad[gs + x];
            if (!(dx - dprev <= tol)) {
                break;
            }
            dprev = dx;
            if (dx - dbase > tol) {
                w.az[gs + base] = zb;
                w.af[gs + base] = fb;
                w.al[gs + base] = lb;
                base = x;
                dbase = dx;
                zb = w.az[gs + x];
                fb = w.af[gs + x];
                lb = w.al[gs + x];
                ++x;
                continue;
            }
            double c, s, r;
            lartg(zb, w.az[gs + x], &c, &s, &r);
            const double fx = w.af[gs + x], lx = w.al[gs + x];
            w.af[gs + x] = -s * fb + c * fx;
            w.al[gs + x] = -s * lb + c * lx;
            fb = c * fb + s * fx;
            lb = c * lb + s * lx;
            zb = r;
            w.az[gs + x] = 0.0;
            w.gmark[gs + x] = 1;
            w.gc[gs + x] = c;
            w.gs[gs + x] = s;
            w.gbase[gs + x] = base;
            ++x;
        }
        w.az[gs + base] = zb;
        w.af[gs + base] = fb;
        w.al[gs + base] = lb;
    }
    __syncthreads();

    // compaction 2: secular poles (padded slice) and rotated-out members
    int carry_p = 0, carry_g = 0;
    double zn = 0.0;
    const long long po = G.poff;
    for (int base = 0; base < Kz; base += 4 * T) {
        int fl[4];
        int cnt = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int idx = base + 4 * threadIdx.x + q;
            fl[q] = (idx < Kz) ? (w.gmark[gs + idx] == 0) : 0;
            cnt += fl[q];
        }
        int tot;
        const int ex = block_exscan<T>(cnt, iscan, &tot);
        int rp = carry_p + ex;
        int rg = carry_g + (4 * threadIdx.x - ex);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int idx = base + 4 * threadIdx.x + q;
            if (idx < Kz) {
                const long long src = gs + idx;
                if (fl[q]) {
                    const long long o = po + rp;
                    const double zv = w.az[src];
                    w.pd[o] = w.ad[src];
                    w.pz[o] = zv;
                    w.pf[o] = w.af[src];
                    w.pl[o] = w.al[src];
                    w.pmap[o] = idx;
                    zn += zv * zv;
                    ++rp;
                } else {
                    const long long o = gs + rg;
                    w.gd[o] = w.ad[src];
                    w.gf[o] = w.af[src];
                    w.gl[o] = w.al[src];
                    ++rg;
                }
            }
        }
        const int valid = (Kz - base) < 4 * T ? (Kz - base) : 4 * T;
        carry_p += tot;
        carry_g += valid - tot;
    }
    const int K = carry_p;
    zn = block_sum<T>(zn, red);

    if (threadIdx.x == 0) {
        w.nK[g] = K;
        w.nKz[g] = Kz;
        w.nrho[g] = rho;
        w.ntol[g] = tol;
        w.nzn[g] = zn;
        brdc_level_diagnostics *dg = &w.hdr->diag[a.k];
        atomicAdd(&dg->merge_count, 1);
        atomicAdd(&dg->size_sum, m);
        atomicAdd(&dg->dd_before_sum, Kz);
        atomicAdd(&dg->dd_after_sum, K);
        atomicMax(&dg->dd_after_max, K);
        atomicAdd(reinterpret_cast<unsigned long long *>(&dg->dd_after_sq_sum),
                  (unsigned long long)K * (unsigned long long)K);
        __threadfence();
        const int t = atomicAdd(&w.hdr->lvl[a.k].ticket, 1);
        s_last = (t == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) {
        return;
    }
    // Last CTA of the level: work plan of the sweep kernels.
    __threadfence();
    long long tk = 0;
    for (int i = threadIdx.x; i < a.nodes; i += T) {
        tk += ((volatile int *)w.nK)[i];
    }
    const double totk = block_sum<T>((double)tk, red);
    const double target = 148.0 * 2048.0;
    int tpr = 1;
    while (tpr < 32 && (double)tpr * totk < target) {
        tpr <<= 1;
    }
    const int R = kSweepThreads / tpr;
    int carry_s = 0, carry_r = 0;
    for (int base = 0; base < a.nodes; base += T) {
        const int i = base + threadIdx.x;
        int is = 0, ir = 0;
        if (i < a.nodes) {
            const int kk = ((volatile int *)w.nK)[i];
            const NodeGeom Gi = node_geom(a.F, a.k, i);
            is = (kk + R - 1) / R;
            ir = (Gi.m + R - 1) / R;
        }
        int ts, tr;
        const int es = block_exscan<T>(is, iscan, &ts);
        const int er = block_exscan<T>(ir, iscan, &tr);
        if (i < a.nodes) {
            w.pref_sec[i] = carry_s + es;
            w.pref_rows[i] = carry_r + er;
        }
        carry_s += ts;
        carry_r += tr;
    }
    if (threadIdx.x == 0) {
        w.pref_sec[a.nodes] = carry_s;
        w.pref_rows[a.nodes] = carry_r;
        LevelCtl *c = &w.hdr->lvl[a.k];
        c->tpr = tpr;
        c->items_sec = carry_s;
        c->items_rows = carry_r;
        c->total_k = (int)totk;
        w.hdr->diag[a.k].threads_per_root = tpr;
    }
}

// ------------------------------------------------------------ sweep tiles
// NA arrays of one node slice staged tile by tile in shared memory with
// cp.async.bulk; two stages.  When the slice fits in the two stages it is
// loaded once and kept resident across sweeps.
template <int NA>
struct TileSet {
    double *buf[2][NA];
    uint64_t *bar;
    unsigned phase[2];
    const double *src[NA];
    long long poff;
    int count;   // elements in the slice
    int ntiles;
    bool resident;
    bool loaded;
};

template <int NA>
__device__ inline void tiles_issue(TileSet<NA> &ts, int stage, int tile) {
    if (threadIdx.x == 0) {
        const int first = tile * kTile;
        int cnt = ts.count - first;
        cnt = cnt < kTile ? cnt : kTile;
        const unsigned bytes = (unsigned)(((cnt + 1) & ~1) * sizeof(double));
        fence_proxy_async();
        mbar_expect_tx(&ts.bar[stage], bytes * NA);
#pragma unroll
        for (int q = 0; q < NA; ++q) {
            bulk_g2s(ts.buf[stage][q], ts.src[q] + ts.poff + first, bytes,
                     &ts.bar[stage]);
        }
    }
}

// Runs one sweep over the slice; body(j0, cnt, bufs) consumes a tile whose
// first element has index j0.  Returns false on a barrier timeout.
template <int NA, typename Body>
__device__ inline bool tiles_sweep(TileSet<NA> &ts, Body body) {
    if (ts.resident) {
        if (!ts.loaded) {
            tiles_issue(ts, 0, 0);
            if (ts.ntiles > 1) {
                tiles_issue(ts, 1, 1);
            }
            bool ok = mbar_wait(&ts.bar[0], ts.phase[0]);
            ts.phase[0] ^= 1u;
            if (ts.ntiles > 1) {
                ok = mbar_wait(&ts.bar[1], ts.phase[1]) && ok;
                ts.phase[1] ^= 1u;
            }
            if (!__syncthreads_and(ok)) {
                return false;
            }
            ts.loaded = true;
        }
        for (int t = 0; t < ts.ntiles; ++t) {
            const int first = t * kTile;
            const int cnt = (ts.count - first) < kTile ? (ts.count - first) : kTile;
            body(first, cnt, ts.buf[t]);
        }
        return true;
    }
    tiles_issue(ts, 0, 0);
    tiles_issue(ts, 1, 1);
    for (int t = 0; t < ts.ntiles; ++t) {
        const int st = t & 1;
        const bool ok = mbar_wait(&ts.bar[st], ts.phase[st]);
        ts.phase[st] ^= 1u;
        if (!__syncthreads_and(ok)) {
            return false;
        }
        const int first = t * kTile;
        const int cnt = (ts.count - first) < kTile ? (ts.count - first) : kTile;
        body(first, cnt, ts.buf[st]);
        __syncthreads();
        if (t + 2 < ts.ntiles) {
            tiles_issue(ts, st, t + 2);
        }
    }
    return true;
}

template <int NA>
__device__ inline void tiles_setup(TileSet<NA> &ts, double *smem, uint64_t *bar,
                                   const double *const *src, long long poff,
                                   int count) {
#pragma unroll
    for (int st = 0; st < 2; ++st) {
#pragma unroll
        for (int q = 0; q < NA; ++q) {
            ts.buf[st][q] = smem + (size_t)(st * NA + q) * kTile;
        }
    }
#pragma unroll
    for (int q = 0; q < NA; ++q) {
        ts.src[q] = src[q];
    }
    ts.bar = bar;
    ts.poff = poff;
    ts.count = count;
    ts.ntiles = (count + kTile - 1) / kTile;
    ts.resident = ts.ntiles <= 2;
    ts.loaded = false;
}

__device__ inline void record_error(WsHeader *h, int code) {
    atomicCAS(&h->status, 0, code);
}

// Item -> node lookup shared through shared memory.
__device__ inline int item_node(const int *pref, int nodes, int item, int *s_node) {
    __syncthreads();
    if (threadIdx.x == 0) {
        *s_node = upper_bound_int(pref, nodes + 1, item) - 1;
    }
    __syncthreads();
    return *s_node;
}

// ---------------------------------------------------------------- roots
__global__ void __launch_bounds__(kSweepThreads)
    k_secular(KArgs a) {
    extern __shared__ __align__(16) double smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ int s_node;
    const Ws &w = a.w;
    const LevelCtl *ctl = &w.hdr->lvl[a.k];
    const int tpr = ctl->tpr;
    const int R = kSweepThreads / tpr;
    const int items = ctl->items_sec;
    const int grp = threadIdx.x / tpr, lane = threadIdx.x % tpr;
    const double eps = DBL_EPSILON;

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    unsigned ph[2] = {0u, 0u};

    for (int item = blockIdx.x; item < items; item += gridDim.x) {
        const int g = item_node(w.pref_sec, a.nodes, item, &s_node);
        const NodeGeom G = node_geom(a.F, a.k, g);
        const int K = w.nK[g];
        const double rho = w.nrho[g];
        const double zn = w.nzn[g];
        const long long po = G.poff;
        const int r = (item - w.pref_sec[g]) * R + grp;
        const bool active = r < K;
        const double *pd = w.pd + po;
        const double *pz = w.pz + po;

        if (K == 1) {
            if (threadIdx.x == 0) {
                const double z0 = pz[0];
                const double t = rho * z0 * z0;
                w.rorg[po] = 0;
                w.rdo[po] = pd[0];
                w.rtau[po] = t;
                w.rlam[po] = pd[0] + t;
            }
            continue;
        }
        SecRoot st;
        if (active) {
            sec_init(st, r, K, pd, pz, rho, zn);
        } else {
            st.stage = 2;
            st.iter = 0;
            st.failed = 0;
        }
        TileSet<2> ts;
        const double *srcs[2] = {w.pd, w.pz};
        tiles_setup<2>(ts, smem, bars, srcs, po, K);
        ts.phase[0] = ph[0];
        ts.phase[1] = ph[1];
        bool ok = true;
        for (;;) {
            SecSums sum;
            sec_zero(sum);
            const bool live = active && st.stage != 2;
            ok = tiles_sweep<2>(ts, [&](int j0, int cnt, double *const *b) {
                if (live) {
                    const double *bd = b[0];
                    const double *bz = b[1];
                    for (int jj = lane; jj < cnt; jj += tpr) {
                        sec_accum(sum, st, j0 + jj, bd[jj], bz[jj]);
                    }
                }
            });
            if (!ok) {
                break;
            }
            for (int o = tpr >> 1; o > 0; o >>= 1) {
                SecSums other;
                other.psi = __shfl_xor_sync(0xffffffffu, sum.psi, o);
                other.dpsi = __shfl_xor_sync(0xffffffffu, sum.dpsi, o);
                other.phi = __shfl_xor_sync(0xffffffffu, sum.phi, o);
                other.dphi = __shfl_xor_sync(0xffffffffu, sum.dphi, o);
                other.err = __shfl_xor_sync(0xffffffffu, sum.err, o);
                sec_combine(sum, other);
            }
            if (live) {
                sec_after_sweep(st, sum, eps);
            }
            const int done = (!active) || st.stage == 2;
            if (__syncthreads_and(done)) {
                break;
            }
        }
        ph[0] = ts.phase[0];
        ph[1] = ts.phase[1];
        if (!ok) {
            record_error(w.hdr, kErrBarrierTimeout);
            return;
        }
        if (active && lane == 0) {
            const long long o = po + r;
            w.rorg[o] = st.org;
            w.rdo[o] = st.dorg;
            w.rtau[o] = st.tau;
            w.rlam[o] = st.dorg + st.tau;
            brdc_level_diagnostics *dg = &w.hdr->diag[a.k];
            atomicAdd(&dg->secular_iter_sum, st.iter);
            atomicMax(&dg->secular_iter_max, st.iter);
            if (st.failed) {
                atomicAdd(&dg->secular_iter_failed, 1);
                atomicAdd(&w.hdr->nonconv, 1);
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------- Loewner z
// For every pole i:  w_i = sign(z_i) * sqrt(-prod_j delta_i(j) /
// prod_{j != i} (d_i - d_j)),  delta_i(j) = (d_i - d_org(j)) - tau_j: the
// recomputation of cpu/src/dlaed9_br.f:181-266 (WPROD), evaluated with one
// lane group per pole sweeping tiles of the roots.
__global__ void __launch_bounds__(kSweepThreads)
    k_lowner(KArgs a) {
    extern __shared__ __align__(16) double smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ int s_node;
    const Ws &w = a.w;
    const LevelCtl *ctl = &w.hdr->lvl[a.k];
    const int tpr = ctl->tpr;
    const int R = kSweepThreads / tpr;
    const int items = ctl->items_sec;
    const int grp = threadIdx.x / tpr, lane = threadIdx.x % tpr;

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    unsigned ph[2] = {0u, 0u};

    for (int item = blockIdx.x; item < items; item += gridDim.x) {
        const int g = item_node(w.pref_sec, a.nodes, item, &s_node);
        const NodeGeom G = node_geom(a.F, a.k, g);
        if (G.depth == 0) {
            continue; // instance root: no parent needs its rows
        }
        const int K = w.nK[g];
        const long long po = G.poff;
        const int i = (item - w.pref_sec[g]) * R + grp;
        const bool active = i < K;
        const double di = active ? w.pd[po + i] : 0.0;
        double prod = 1.0;
        TileSet<3> ts;
        const double *srcs[3] = {w.rdo, w.rtau, w.pd};
        tiles_setup<3>(ts, smem, bars, srcs, po, K);
        ts.phase[0] = ph[0];
        ts.phase[1] = ph[1];
        const bool ok = tiles_sweep<3>(ts, [&](int j0, int cnt, double *const *b) {
            if (active) {
                for (int jj = lane; jj < cnt; jj += tpr) {
                    const int j = j0 + jj;
                    const double dl = (di - b[0][jj]) - b[1][jj];
                    prod *= (j == i) ? dl : dl / (di - b[2][jj]);
                }
            }
        });
        ph[0] = ts.phase[0];
        ph[1] = ts.phase[1];
        if (!ok) {
            record_error(w.hdr, kErrBarrierTimeout);
            return;
        }
        for (int o = tpr >> 1; o > 0; o >>= 1) {
            prod *= __shfl_xor_sync(0xffffffffu, prod, o);
        }
        if (active && lane == 0) {
            const double zi = w.pz[po + i];
            const double mag = sqrt(fmax(-prod, 0.0));
            double wi = zi < 0.0 ? -mag : mag;
            if (!(mag > 0.0) || !isfinite(mag)) {
                wi = zi * sqrt(w.nrho[g]);
            }
            w.pw[po + i] = wi;
        }
        __syncthreads();
    }
}

// ------------------------------------------------- rows and placement
// Slot s < K is root s: its eigenvector u_i = w_i / delta_i(s), normalised,
// gives new_first = sum_i f_i u_i and new_last = sum_i l_i u_i (the streamed
// update of cpu/src/dlaed9_br.f:272-334 with the compact delta).  Slots
// K.. are the deflated eigenvalues.  Every slot is written to its place in
// the ascending spectrum of the node: roots and the two deflated lists are
// merged by rank (ties: roots, then small-z, then rotated).
__global__ void __launch_bounds__(kSweepThreads)
    k_rows_place(KArgs a) {
    extern __shared__ __align__(16) double smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ int s_node;
    const Ws &w = a.w;
    const LevelCtl *ctl = &w.hdr->lvl[a.k];
    const int tpr = ctl->tpr;
    const int R = kSweepThreads / tpr;
    const int items = ctl->items_rows;
    const int grp = threadIdx.x / tpr, lane = threadIdx.x % tpr;

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    unsigned ph[2] = {0u, 0u};

    for (int item = blockIdx.x; item < items; item += gridDim.x) {
        const int g = item_node(w.pref_rows, a.nodes, item, &s_node);
        const NodeGeom G = node_geom(a.F, a.k, g);
        const int K = w.nK[g];
        const int Kz = w.nKz[g];
        const int m = G.m;
        const int ndz = m - Kz, ndg = Kz - K;
        const long long po = G.poff, gs = G.gstart;
        const int b0 = (item - w.pref_rows[g]) * R;
        const int s = b0 + grp;
        const bool top = (G.depth == 0);
        double a1 = 0.0, a2 = 0.0, s2 = 0.0;
        if (!top && b0 < K) {
            const bool root = s < K;
            const double dorg = root ? w.rdo[po + s] : 0.0;
            const double tau = root ? w.rtau[po + s] : 0.0;
            TileSet<4> ts;
            const double *srcs[4] = {w.pd, w.pw, w.pf, w.pl};
            tiles_setup<4>(ts, smem, bars, srcs, po, K);
            ts.phase[0] = ph[0];
            ts.phase[1] = ph[1];
            const bool ok = tiles_sweep<4>(ts, [&](int j0, int cnt, double *const *b) {
                if (root) {
                    for (int jj = lane; jj < cnt; jj += tpr) {
                        const double dl = (b[0][jj] - dorg) - tau;
                        const double u = (dl != 0.0) ? b[1][jj] / dl : 0.0;
                        s2 += u * u;
                        a1 += b[2][jj] * u;
                        a2 += b[3][jj] * u;
                    }
                }
            });
            ph[0] = ts.phase[0];
            ph[1] = ts.phase[1];
            if (!ok) {
                record_error(w.hdr, kErrBarrierTimeout);
                return;
            }
            for (int o = tpr >> 1; o > 0; o >>= 1) {
                s2 += __shfl_xor_sync(0xffffffffu, s2, o);
                a1 += __shfl_xor_sync(0xffffffffu, a1, o);
                a2 += __shfl_xor_sync(0xffffffffu, a2, o);
            }
        }
        if (s < m && lane == 0) {
            double val, fo = 0.0, lo = 0.0;
            int pos;
            const double *zdl = w.zd + gs;
            const double *gdl = w.gd + gs;
            const double *rl = w.rlam + po;
            if (s < K) {
                val = rl[s];
                pos = s + lower_bound_d(zdl, ndz, val) + lower_bound_d(gdl, ndg, val);
                if (!top) {
                    const double nrm = sqrt(s2);
                    fo = (nrm > 0.0) ? a1 / nrm : 0.0;
                    lo = (nrm > 0.0) ? a2 / nrm : 0.0;
                }
            } else if (s < K + ndz) {
                const int q = s - K;
                val = zdl[q];
                pos = q + upper_bound_d(rl, K, val) + lower_bound_d(gdl, ndg, val);
                fo = w.zf[gs + q];
                lo = w.zl[gs + q];
            } else {
                const int q = s - K - ndz;
                val = gdl[q];
                pos = q + upper_bound_d(rl, K, val) + upper_bound_d(zdl, ndz, val);
                fo = w.gf[gs + q];
                lo = w.gl[gs + q];
            }
            const long long o = gs + pos;
            if (top) {
                a.W[o] = val;
            } else {
                w.nd[o] = val;
                w.nf[o] = fo;
                w.nl[o] = lo;
            }
        }
        __syncthreads();
    }
}

__global__ void k_init(WsHeader *h, int levels, int B, long long total_n,
                       long long leaves, int flags) {
    const int t = threadIdx.x;
    if (t == 0) {
        h->magic = kWsMagic;
        h->B = B;
        h->total_n = total_n;
        h->max_levels = levels;
        h->flags = flags;
        h->leaf_count = (int)leaves;
        h->status = 0;
        h->nonconv = 0;
        h->leaf_sweeps_max = 0;
    }
    for (int k = t; k < BRDC_MAX_LEVELS; k += blockDim.x) {
        h->lvl[k].ticket = 0;
        h->lvl[k].tpr = 1;
        h->lvl[k].items_sec = 0;
        h->lvl[k].items_rows = 0;
        h->lvl[k].total_k = 0;
        brdc_level_diagnostics z = {};
        z.level = k;
        h->diag[k] = z;
    }
}

} // namespace brdc
