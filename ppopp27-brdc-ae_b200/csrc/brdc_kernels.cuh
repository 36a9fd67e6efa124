// brdc_kernels.cuh -- sm_100a kernels of the forward BR solve.
//
// A forest level solved by per-level kernels (the levels the fused level
// kernel of brdc_level.cuh does not take) runs:
//   k_merge          one thread per row: rank merge of the two sorted child
//                    spectra, z from the children's boundary rows
//   k_merge_deflate  one CTA (or a cluster of CTAs) per merge: small-z and
//                    close-pole deflation with Givens rotations of z and of
//                    both boundary rows, compaction, work plan of the level
//   k_sweeps         one cooperative launch, its phases separated by grid
//                    barriers:
//     secular        secular roots, TPR lanes per root; merges with K <=
//                    kWarpMaxK one warp per work item (poles through L1),
//                    larger ones one CTA per item with pole tiles staged in
//                    shared memory by cp.async.bulk
//     Loewner        Loewner / Gu-Eisenstat recomputation of z (same roles)
//     rows           first/last rows of the merged eigenvector matrix for
//                    every root (same roles)
//     placement      one thread per row: every eigenvalue of a node to its
//                    place in the node's ascending spectrum
// The leaves are solved first by k_leaf (one warp per two leaves, parallel
// cyclic Jacobi) or inside k_subtree.
#pragma once

#include <cooperative_groups.h>

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
    long long level_rows; // rows of the instances that merge at this level
    int plan_inline;    // the last deflation CTA writes the level plan (else k_plan)
    int lanes_target;   // threads the root sweeps aim to keep busy
    int big_k;          // > 0: the plan and the placement serve only nodes with
                        // K > big_k (k_level finished the others)
};

// ------------------------------------------------------------------ leaves
// Leaves of <= 16 rows, two per warp (one per half-warp), by parallel
// cyclic Jacobi, as the reference solves its leaves by Jacobi
// (gpu/src/tridiag_solver_leaf.cuh:56-123, one thread per leaf there).
//
// Lane x of a half-warp owns column x of the 16x16 leaf matrix in
// registers, stored XOR-skewed: reg[j] = A[x^j][x].  Sweep m = 1..15 of the
// XOR tournament pairs index x with x^m (every pair exactly once per sweep),
// so in round m: the diagonal is reg[0], the entry to annihilate is reg[m],
// the two rows a rotation mixes in my column are reg[j] and reg[j^m], and
// the partner column's entry of the same row is the partner lane's
// reg[j^m] -- all compile-time register indices, exchanged by
// __shfl_xor_sync.  Only the first and last rows of the eigenvector matrix
// are accumulated (two values per lane).  The rank-one cut corrections
// D -= |E_cut| at both ends (gpu/src/tridiag_solver_extract.cuh:104-117) are
// applied on load.  Output: ascending eigenvalues with the first and last
// rows in that order.
constexpr int kLeafWarps = 4;
constexpr unsigned kFull = 0xffffffffu;

// The arithmetic of a leaf rotation, spelled out (explicit FMAs and rounded
// products, nothing left for the compiler to contract), so that leaf_round
// and leaf_round_v produce bit for bit the same matrix and rows.
__device__ __forceinline__ double leaf_rot(double c, double x, double sgs, double y) {
    return fma(c, x, __dmul_rn(sgs, y)); // c x + (sg s) y
}

template <int M>
__device__ __forceinline__ void leaf_round(double (&a)[16], double &v0,
                                           double &v1, int x, double th) {
    const bool isp = x < (x ^ M);
    const double mydiag = a[0];
    const double odiag = __shfl_xor_sync(kFull, mydiag, M);
    // both lanes of a pair compute the rotation from the same three numbers
    // (the lower column's off-diagonal entry), so both columns turn by
    // exactly the same plane rotation without exchanging it
    const double apq_mine = a[M];
    const double apq_o = __shfl_xor_sync(kFull, apq_mine, M);
    const double apq = isp ? apq_mine : apq_o;
    const double app = isp ? mydiag : odiag;
    const double aqq = isp ? odiag : mydiag;
    double c = 1.0, sn = 0.0, t = 0.0;
    int rot = 0;
    if (fabs(apq) > th) {
        const double theta = (aqq - app) / (2.0 * apq);
        if (fabs(theta) > 1.0e150) {
            t = 0.5 / theta;
        } else {
            t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(fma(theta, theta, 1.0)));
        }
        c = 1.0 / sqrt(fma(t, t, 1.0));
        sn = __dmul_rn(t, c);
        rot = 1;
    }
    // columns: B = A J  (col p: c*col_p - s*col_q, col q: s*col_p + c*col_q)
    const double sgx = isp ? -1.0 : 1.0;
    double b[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const double other = __shfl_xor_sync(kFull, a[j ^ M], M);
        b[j] = leaf_rot(c, a[j], __dmul_rn(sgx, sn), other);
    }
    {
        const double o0 = __shfl_xor_sync(kFull, v0, M);
        const double o1 = __shfl_xor_sync(kFull, v1, M);
        v0 = leaf_rot(c, v0, __dmul_rn(sgx, sn), o0);
        v1 = leaf_rot(c, v1, __dmul_rn(sgx, sn), o1);
    }
    // rows: A' = J^T B; rows x^j and x^j^M use the rotation of lane x^j
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if (j < (j ^ M)) {
            const int jj = j ^ M;
            const double cr = __shfl_xor_sync(kFull, c, j);
            const double sr = __shfl_xor_sync(kFull, sn, j);
            const int r = x ^ j;
            const double sgr = (r < (r ^ M)) ? -1.0 : 1.0;
            const double bj = b[j], bjj = b[jj];
            a[j] = leaf_rot(cr, bj, __dmul_rn(sgr, sr), bjj);
            a[jj] = leaf_rot(cr, bjj, -__dmul_rn(sgr, sr), bj);
        }
    }
    if (rot) {
        a[0] = isp ? fma(-t, apq, app) : fma(t, apq, aqq);
        a[M] = 0.0;
    }
}

__device__ __forceinline__ double half_max(double v) {
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
        v = fmax(v, __shfl_xor_sync(kFull, v, o));
    }
    return v;
}

// Jacobi solve of one leaf by a half-warp (lane x of the half owns column x;
// both halves of the warp call this together, the other half on its own
// leaf or with s = 0).  Returns the leaf's eigenvalue of rank x (ascending;
// +inf for x >= s) with the first and last entries of its eigenvector, and
// the number of sweeps taken.
__device__ inline int leaf_solve(const KArgs &a, const LeafGeom &G, int s, int x,
                                 double *key_out, double *v0_out, double *v1_out) {
    const double eps = DBL_EPSILON;
    double dx = 0.0, ex = 0.0, exm1 = 0.0;
    if (x < s) {
        const double sc = inst_scale(a.w, G.inst);
        dx = sc * a.D[G.gstart + x];
        if (x == 0 && G.gstart > G.istart) {
            dx -= sc * fabs(a.E[G.gstart - 1]);
        }
        if (x == s - 1 && G.gstart + s < G.iend) {
            dx -= sc * fabs(a.E[G.gstart + s - 1]);
        }
        if (x + 1 < s) {
            ex = sc * fabs(a.E[G.gstart + x]);
        }
        if (x >= 1) {
            exm1 = sc * fabs(a.E[G.gstart + x - 1]);
        }
    }
    double reg[16];
    const int jup = x ^ (x + 1);
    const int jdn = x ^ (x - 1);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        reg[j] = (j == 0) ? dx : ((j == jup) ? ex : ((j == jdn) ? exm1 : 0.0));
    }
    double v0 = (x == 0 && s > 0) ? 1.0 : 0.0;
    double v1 = (x == s - 1) ? 1.0 : 0.0;
    const double amax = half_max(fmax(fabs(dx), fmax(ex, exm1)));
    // Sweeps stop, and rotations are skipped, once an off-diagonal entry is
    // at most eps max|T_leaf|: what it leaves in an eigenvalue is of the
    // order of its rounding.  A threshold 1000 times smaller cost 3% more
    // sweeps on B200 (uniform 65,536) and changed no tested result.
    const double th = eps * amax;
    int sweep = 0;
    for (; sweep < 40; ++sweep) {
        double off = 0.0;
#pragma unroll
        for (int j = 1; j < 16; ++j) {
            off = fmax(off, fabs(reg[j]));
        }
        off = half_max(off);
        if (!__any_sync(kFull, off > th)) {
            break;
        }
        leaf_round<1>(reg, v0, v1, x, th);
        leaf_round<2>(reg, v0, v1, x, th);
        leaf_round<3>(reg, v0, v1, x, th);
        leaf_round<4>(reg, v0, v1, x, th);
        leaf_round<5>(reg, v0, v1, x, th);
        leaf_round<6>(reg, v0, v1, x, th);
        leaf_round<7>(reg, v0, v1, x, th);
        leaf_round<8>(reg, v0, v1, x, th);
        leaf_round<9>(reg, v0, v1, x, th);
        leaf_round<10>(reg, v0, v1, x, th);
        leaf_round<11>(reg, v0, v1, x, th);
        leaf_round<12>(reg, v0, v1, x, th);
        leaf_round<13>(reg, v0, v1, x, th);
        leaf_round<14>(reg, v0, v1, x, th);
        leaf_round<15>(reg, v0, v1, x, th);
    }

    // bitonic sort of (eigenvalue, column) within the half-warp
    double key = (x < s) ? reg[0] : INFINITY;
    int col = x;
#pragma unroll
    for (int size = 2; size <= 16; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const double ok = __shfl_xor_sync(kFull, key, stride);
            const int oc = __shfl_xor_sync(kFull, col, stride);
            const double o0 = __shfl_xor_sync(kFull, v0, stride);
            const double o1 = __shfl_xor_sync(kFull, v1, stride);
            const bool up = (size == 16) || ((x & size) == 0);
            const bool lower = ((x & stride) == 0);
            const bool take_min = (up == lower);
            const bool swap = take_min ? (ok < key || (ok == key && oc < col))
                                       : (ok > key || (ok == key && oc > col));
            if (swap) {
                key = ok;
                col = oc;
                v0 = o0;
                v1 = o1;
            }
        }
    }
    *key_out = key;
    *v0_out = v0;
    *v1_out = v1;
    return sweep;
}

// leaf_round on the whole eigenvector matrix (lane x holds column x in v):
// the same rotation, applied to every row with leaf_round's arithmetic.
template <int M>
__device__ __forceinline__ void leaf_round_v(double (&a)[16], double (&v)[16],
                                             int x, double th) {
    const bool isp = x < (x ^ M);
    const double mydiag = a[0];
    const double odiag = __shfl_xor_sync(kFull, mydiag, M);
    // both lanes of a pair compute the rotation from the same three numbers
    // (the lower column's off-diagonal entry), so both columns turn by
    // exactly the same plane rotation without exchanging it
    const double apq_mine = a[M];
    const double apq_o = __shfl_xor_sync(kFull, apq_mine, M);
    const double apq = isp ? apq_mine : apq_o;
    const double app = isp ? mydiag : odiag;
    const double aqq = isp ? odiag : mydiag;
    double c = 1.0, sn = 0.0, t = 0.0;
    int rot = 0;
    if (fabs(apq) > th) {
        const double theta = (aqq - app) / (2.0 * apq);
        if (fabs(theta) > 1.0e150) {
            t = 0.5 / theta;
        } else {
            t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(fma(theta, theta, 1.0)));
        }
        c = 1.0 / sqrt(fma(t, t, 1.0));
        sn = __dmul_rn(t, c);
        rot = 1;
    }
    const double sgx = isp ? -1.0 : 1.0;
    double b[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const double other = __shfl_xor_sync(kFull, a[j ^ M], M);
        b[j] = leaf_rot(c, a[j], __dmul_rn(sgx, sn), other);
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const double other = __shfl_xor_sync(kFull, v[j], M);
        v[j] = leaf_rot(c, v[j], __dmul_rn(sgx, sn), other);
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if (j < (j ^ M)) {
            const int jj = j ^ M;
            const double cr = __shfl_xor_sync(kFull, c, j);
            const double sr = __shfl_xor_sync(kFull, sn, j);
            const int r = x ^ j;
            const double sgr = (r < (r ^ M)) ? -1.0 : 1.0;
            const double bj = b[j], bjj = b[jj];
            a[j] = leaf_rot(cr, bj, __dmul_rn(sgr, sr), bjj);
            a[jj] = leaf_rot(cr, bjj, -__dmul_rn(sgr, sr), bj);
        }
    }
    if (rot) {
        a[0] = isp ? fma(-t, apq, app) : fma(t, apq, aqq);
        a[M] = 0.0;
    }
}

// leaf_solve with the whole eigenvector matrix, for a checkpointing
// forward (the adjoint of a leaf needs all of it): the same sweeps and
// rotations, so rows 0 and s-1 of v are bit for bit leaf_solve's v0 and v1,
// and the same sort.  Lane x returns the eigenvalue of rank x and its
// eigenvector (rows 0..15, zero past s).
__device__ inline int leaf_solve_full(const KArgs &a, const LeafGeom &G, int s, int x,
                                      double *key_out, double (&v)[16]) {
    const double eps = DBL_EPSILON;
    double dx = 0.0, ex = 0.0, exm1 = 0.0;
    if (x < s) {
        const double sc = inst_scale(a.w, G.inst);
        dx = sc * a.D[G.gstart + x];
        if (x == 0 && G.gstart > G.istart) {
            dx -= sc * fabs(a.E[G.gstart - 1]);
        }
        if (x == s - 1 && G.gstart + s < G.iend) {
            dx -= sc * fabs(a.E[G.gstart + s - 1]);
        }
        if (x + 1 < s) {
            ex = sc * fabs(a.E[G.gstart + x]);
        }
        if (x >= 1) {
            exm1 = sc * fabs(a.E[G.gstart + x - 1]);
        }
    }
    double reg[16];
    const int jup = x ^ (x + 1);
    const int jdn = x ^ (x - 1);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        reg[j] = (j == 0) ? dx : ((j == jup) ? ex : ((j == jdn) ? exm1 : 0.0));
        v[j] = (j == x) ? 1.0 : 0.0;
    }
    const double amax = half_max(fmax(fabs(dx), fmax(ex, exm1)));
    const double th = eps * amax;
    int sweep = 0;
    for (; sweep < 40; ++sweep) {
        double off = 0.0;
#pragma unroll
        for (int j = 1; j < 16; ++j) {
            off = fmax(off, fabs(reg[j]));
        }
        off = half_max(off);
        if (!__any_sync(kFull, off > th)) {
            break;
        }
        leaf_round_v<1>(reg, v, x, th);
        leaf_round_v<2>(reg, v, x, th);
        leaf_round_v<3>(reg, v, x, th);
        leaf_round_v<4>(reg, v, x, th);
        leaf_round_v<5>(reg, v, x, th);
        leaf_round_v<6>(reg, v, x, th);
        leaf_round_v<7>(reg, v, x, th);
        leaf_round_v<8>(reg, v, x, th);
        leaf_round_v<9>(reg, v, x, th);
        leaf_round_v<10>(reg, v, x, th);
        leaf_round_v<11>(reg, v, x, th);
        leaf_round_v<12>(reg, v, x, th);
        leaf_round_v<13>(reg, v, x, th);
        leaf_round_v<14>(reg, v, x, th);
        leaf_round_v<15>(reg, v, x, th);
    }
    // bitonic sort of (eigenvalue, column) within the half-warp, as leaf_solve
    double key = (x < s) ? reg[0] : INFINITY;
    int col = x;
#pragma unroll
    for (int size = 2; size <= 16; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const double ok = __shfl_xor_sync(kFull, key, stride);
            const int oc = __shfl_xor_sync(kFull, col, stride);
            double ov[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                ov[j] = __shfl_xor_sync(kFull, v[j], stride);
            }
            const bool up = (size == 16) || ((x & size) == 0);
            const bool lower = ((x & stride) == 0);
            const bool take_min = (up == lower);
            const bool swap = take_min ? (ok < key || (ok == key && oc < col))
                                       : (ok > key || (ok == key && oc > col));
            if (swap) {
                key = ok;
                col = oc;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    v[j] = ov[j];
                }
            }
        }
    }
    *key_out = key;
    return sweep;
}

// The leaves of a checkpointing forward: leaf_solve_full, then the leaf
// outputs as k_leaf writes them plus, for the adjoint, every eigenvalue
// (leafl) and eigenvector (leafv, 16 entries per column) in sorted order.
__global__ void __launch_bounds__(kLeafWarps * 32)
    k_leaf_full(KArgs a, long long total_leaves) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    const int lane = threadIdx.x & 31;
    const int x = lane & 15;
    const int half = lane >> 4;
    int sweeps_max = 0, sweeps_sum = 0;
    const long long pairs = (total_leaves + 1) / 2;
    for (long long pr = (long long)blockIdx.x * kLeafWarps + (threadIdx.x >> 5); pr < pairs;
         pr += (long long)gridDim.x * kLeafWarps) {
        const long long leaf = 2 * pr + half;
        const bool has = leaf < total_leaves;
        LeafGeom G{};
        int s = 0;
        if (has) {
            G = leaf_geom(a.F, leaf);
            s = G.s;
        }
        double key, v[16];
        const int sweep = leaf_solve_full(a, G, s, x, &key, v);
        sweeps_max = sweeps_max > sweep ? sweeps_max : sweep;
        sweeps_sum += (x == 0 && s > 0) ? sweep : 0;
        if (x < s) {
            const long long o = G.gstart + x;
            double vlast = 0.0;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                vlast = (j == s - 1) ? v[j] : vlast;
                a.w.leafv[o * 16 + j] = (j < s) ? v[j] : 0.0;
            }
            a.w.leafl[o] = key;
            if (G.top) {
                a.W[o] = key * inst_unscale(a.w, G.inst);
            } else {
                a.w.cd[o] = key;
                a.w.cf[o] = v[0];
                a.w.cl[o] = vlast;
            }
        }
    }
    sweeps_sum = __reduce_add_sync(kFull, sweeps_sum);
    if (lane == 0 && sweeps_max > 0) {
        atomicMax(&a.w.hdr->leaf_sweeps_max, sweeps_max);
        atomicAdd(&a.w.hdr->leaf_sweeps_sum, sweeps_sum);
    }
}

__global__ void __launch_bounds__(kLeafWarps * 32)
    k_leaf(KArgs a, long long total_leaves) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    const int lane = threadIdx.x & 31;
    const int x = lane & 15;
    const int half = lane >> 4;
    int sweeps_max = 0, sweeps_sum = 0;
    const long long pairs = (total_leaves + 1) / 2;
    for (long long pr = (long long)blockIdx.x * kLeafWarps + (threadIdx.x >> 5); pr < pairs;
         pr += (long long)gridDim.x * kLeafWarps) {
        const long long leaf = 2 * pr + half;
        const bool has = leaf < total_leaves;
        LeafGeom G{};
        int s = 0;
        if (has) {
            G = leaf_geom(a.F, leaf);
            s = G.s;
        }
        double key, v0, v1;
        const int sweep = leaf_solve(a, G, s, x, &key, &v0, &v1);
        sweeps_max = sweeps_max > sweep ? sweeps_max : sweep;
        sweeps_sum += (x == 0 && s > 0) ? sweep : 0;
        if (x < s) {
            const long long o = G.gstart + x;
            if (G.top) {
                a.W[o] = key * inst_unscale(a.w, G.inst);
            } else {
                a.w.cd[o] = key;
                a.w.cf[o] = v0;
                a.w.cl[o] = v1;
            }
        }
    }
    sweeps_sum = __reduce_add_sync(kFull, sweeps_sum);
    if (lane == 0 && sweeps_max > 0) {
        atomicMax(&a.w.hdr->leaf_sweeps_max, sweeps_max);
        atomicAdd(&a.w.hdr->leaf_sweeps_sum, sweeps_sum);
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
// Rank merge of the two sorted child spectra of every merge of the level,
// one thread per row: a row of the left child lands at its own index plus
// the number of right-child poles below it, a right-child row at its index
// plus the left-child poles at or below it (left wins ties).  Writes the
// merged d, z = (last row of the left child | first row of the right
// child)/sqrt2, and the block-diagonal projections of the parent's first
// and last rows.
__global__ void __launch_bounds__(256) k_merge(KArgs a, long long total_n) {
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
        const int m1 = m >> 1, m2 = m - m1;
        const int e = (int)(x - gs);
        const double *Ad = w.cd + gs;
        const double *Bd = w.cd + gs + m1;
        double xv, z, f, l;
        int pos;
        if (e < m1) {
            xv = Ad[e];
            pos = e + lower_bound_d(Bd, m2, xv);
            z = w.cl[x] / kSqrt2;
            f = w.cf[x];
            l = 0.0;
        } else {
            const int j = e - m1;
            xv = Bd[j];
            pos = j + upper_bound_d(Ad, m1, xv);
            z = w.cf[x] / kSqrt2;
            f = 0.0;
            l = w.cl[x];
        }
        const long long o = gs + pos;
        w.md[o] = xv;
        w.mz[o] = z;
        w.mf[o] = f;
        w.ml[o] = l;
        w.morig[o] = e;
    }
}

// Work plan of the sweep kernels for level a.k, from the node scalars the
// deflation wrote: the level diagnostics, lanes per root, and the item
// tables.  Merges with K <= kWarpMaxK are served one warp per work item;
// larger ones by whole CTAs that stage pole tiles in shared memory.  Run by
// the last deflation CTA of the level, or by k_plan where the level has
// many nodes and that CTA would be narrow.
template <int T>
__device__ void level_plan(const KArgs &a, double *red, int *iscan) {
    const Ws &w = a.w;
    double tkw = 0.0, tkc = 0.0, cw = 0.0, cc = 0.0, qw = 0.0, qc = 0.0;
    double skz = 0.0, sk = 0.0, sk2 = 0.0, kmax = 0.0;
    for (int i = threadIdx.x; i < a.nodes; i += T) {
        const int kk = __ldcg(w.nK + i);
        const int kz = __ldcg(w.nKz + i);
        // nodes with K <= big_k get no items (finished by k_level, or empty)
        if (kk > a.big_k && kk > kWarpMaxK) {
            tkc += kk;
            cc += 1.0;
            qc += (double)kk * (double)kk;
        } else if (kk > a.big_k) {
            tkw += kk;
            cw += 1.0;
            qw += (double)kk * (double)kk;
        }
        skz += kz;
        sk += kk;
        sk2 += (double)kk * (double)kk;
        kmax = fmax(kmax, (double)kk);
    }
    tkw = block_sum<T>(tkw, red);
    tkc = block_sum<T>(tkc, red);
    cw = block_sum<T>(cw, red);
    cc = block_sum<T>(cc, red);
    qw = block_sum<T>(qw, red);
    qc = block_sum<T>(qc, red);
    skz = block_sum<T>(skz, red);
    sk = block_sum<T>(sk, red);
    sk2 = block_sum<T>(sk2, red);
    kmax = block_max<T>(kmax, red);
    if (threadIdx.x == 0) {
        // level counters of the reference's diagnostics
        // (gpu/src/tridiag_solver.cu:1166-1260), gathered once per level
        brdc_level_diagnostics *dg = &w.hdr->diag[a.k];
        dg->merge_count = a.nodes;
        dg->size_sum = (int)(a.level_rows);
        dg->dd_before_sum = (int)skz;
        dg->dd_after_sum = (int)(sk);
        dg->dd_after_max = (int)kmax;
        dg->dd_after_sq_sum = (long long)sk2;
    }
    // warp role: each root's sweeps form a serial latency chain, so spread
    // the roots over enough lanes to keep every scheduler busy (by default
    // ~75k threads); with one root per warp the warp also never diverges.
    int tpr_w = 1;
    while (tpr_w < 32 && (double)tpr_w * tkw < (double)a.lanes_target) {
        tpr_w <<= 1;
    }
    // CTA role: enough lanes to fill the GPU, at least ~16 poles per lane
    // and sweep
    const double kavg_c = tkc / fmax(cc, 1.0);
    int tpr_c = 1;
    while (tpr_c < 32 && (double)tpr_c * tkc < (double)a.lanes_target) {
        tpr_c <<= 1;
    }
    int cap = 1;
    while (cap < 32 && (double)(cap * 2) * 16.0 <= kavg_c) {
        cap <<= 1;
    }
    tpr_c = tpr_c < cap ? tpr_c : cap;
    const int Rw = 32 / tpr_w;
    const int Rc = kSweepThreads / tpr_c;
    // each thread owns a contiguous run of nodes: serial prefix of its run,
    // one block scan across threads, then the run's prefixes
    const int per = (a.nodes + T - 1) / T;
    const int i0 = threadIdx.x * per;
    const int i1 = (i0 + per < a.nodes) ? i0 + per : a.nodes;
    int sw = 0, sc = 0;
    for (int i = i0; i < i1; ++i) {
        const int kk = __ldcg(w.nK + i);
        if (kk > a.big_k && kk > kWarpMaxK) {
            sc += (kk + Rc - 1) / Rc;
        } else if (kk > a.big_k) {
            sw += (kk + Rw - 1) / Rw;
        }
    }
    int carry_w, carry_c;
    int rw = block_exscan<T>(sw, iscan, &carry_w);
    int rc = block_exscan<T>(sc, iscan, &carry_c);
    for (int i = i0; i < i1; ++i) {
        const int kk = __ldcg(w.nK + i);
        w.pref_w[i] = rw;
        w.pref_c[i] = rc;
        if (kk > a.big_k && kk > kWarpMaxK) {
            rc += (kk + Rc - 1) / Rc;
        } else if (kk > a.big_k) {
            rw += (kk + Rw - 1) / Rw;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < a.nodes; i += T) {
        const int s0 = w.pref_w[i];
        const int s1 = (i + 1 < a.nodes) ? w.pref_w[i + 1] : carry_w;
        for (int q = s0; q < s1; ++q) {
            w.items_w[q] = i;
        }
        const int c0 = w.pref_c[i];
        const int c1 = (i + 1 < a.nodes) ? w.pref_c[i + 1] : carry_c;
        for (int q = c0; q < c1; ++q) {
            w.items_c[q] = i;
        }
    }
    if (threadIdx.x == 0) {
        w.pref_w[a.nodes] = carry_w;
        w.pref_c[a.nodes] = carry_c;
        LevelCtl *c = &w.hdr->lvl[a.k];
        c->tpr_w = tpr_w;
        c->tpr_c = tpr_c;
        c->items_w = carry_w;
        c->items_c = carry_c;
        c->total_k = (int)(tkw + tkc);
        c->work_w = qw;
        c->work_c = qc;
        w.hdr->diag[a.k].threads_per_root = carry_c > 0 ? tpr_c : tpr_w;
    }
}

template <int T>
__global__ void __launch_bounds__(T) k_plan(KArgs a) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    __shared__ double red[32];
    __shared__ int iscan[32];
    level_plan<T>(a, red, iscan);
}

// The full plans (every merge) of many levels in one launch, one CTA per
// level: what a checkpointed forward leaves for the adjoint's sweeps on the
// levels it solved without them (subtree and fused levels).  A level's plan
// reads and writes only these arrays of its workspace slice.
struct PlanLevel {
    int *nK, *nKz, *pref_w, *pref_c, *items_w, *items_c;
    int nodes, k;
    long long rows;
};
constexpr int kPlanMaxLevels = 40;
struct PlanAllArgs {
    KArgs base;
    PlanLevel lv[kPlanMaxLevels];
};

template <int T>
__global__ void __launch_bounds__(T) k_plan_all(PlanAllArgs P) {
    pdl_begin();
    if (halted(P.base.w.hdr)) {
        return;
    }
    __shared__ double red[32];
    __shared__ int iscan[32];
    const PlanLevel &L = P.lv[blockIdx.x];
    KArgs a = P.base;
    a.w.nK = L.nK;
    a.w.nKz = L.nKz;
    a.w.pref_w = L.pref_w;
    a.w.pref_c = L.pref_c;
    a.w.items_w = L.items_w;
    a.w.items_c = L.items_c;
    a.nodes = L.nodes;
    a.level_rows = L.rows;
    a.k = L.k;
    a.big_k = 0;
    level_plan<T>(a, red, iscan);
}

constexpr int kDeflEPT = 4; // rows per thread per deflation chunk

// Deflation phases over a range of rows, shared by the one-CTA-per-node
// kernel (whole node) and the cluster kernel (one slice per CTA).

// Chunks of EPT*T rows: warp w of the CTA takes rows [w*128, w*128+128) of
// the chunk, lane l rows w*128 + 32q + l (q < EPT), so every load is one
// coalesced 256-byte row of the warp.  Order is kept by warp ballots: the
// rank of a row among the chunk's survivors is the survivors of the warps
// before it (one block scan of the warp totals) plus those of its own warp
// before it (popcounts of the EPT ballots).

// Exclusive prefix of this warp's count over the CTA's warps, and the total.
template <int T>
__device__ inline int defl_warp_prefix(int wcnt, int *iscan, int *total) {
    const int lane = threadIdx.x & 31;
    const int ex = block_exscan<T>(lane == 0 ? wcnt : 0, iscan, total);
    return __shfl_sync(0xffffffffu, ex, 0);
}

// Rows [r0, r1) of the merged node that survive the small-z test.
template <int T>
__device__ int defl_count_active(const Ws &w, long long gs, int r0, int r1, double rho,
                                 double tol, int *iscan) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int wcnt = 0;
    for (int base = r0; base < r1; base += kDeflEPT * T) {
        const int wbase = base + wid * (kDeflEPT * 32);
#pragma unroll
        for (int q = 0; q < kDeflEPT; ++q) {
            const int idx = wbase + 32 * q + lane;
            const bool f = idx < r1 && fabs(rho * w.mz[gs + idx]) > tol;
            wcnt += __popc(__ballot_sync(0xffffffffu, f));
        }
    }
    int tot;
    defl_warp_prefix<T>(wcnt, iscan, &tot);
    return tot;
}

// Compaction 1 of rows [r0, r1): small-z survivors to the active list from
// position carry_a, deflated rows to the small-z list from carry_z, both in
// merged order.  Every value a thread moves is loaded before the scan, so a
// chunk costs one round trip to L2.  Returns carry_a plus the survivors.
template <int T>
__device__ int defl_compact_active(const Ws &w, long long gs, int r0, int r1, double rho,
                                   double tol, int carry_a, int carry_z, int *iscan) {
    constexpr int EPT = kDeflEPT;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (int base = r0; base < r1; base += EPT * T) {
        const int wbase = base + wid * (EPT * 32);
        bool fl[EPT];
        unsigned bal[EPT];
        double vd[EPT], vz[EPT], vf[EPT], vl[EPT];
        int wcnt = 0;
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            const int idx = wbase + 32 * q + lane;
            const bool ok = idx < r1;
            const long long src = gs + (ok ? idx : r0);
            vd[q] = w.md[src];
            vz[q] = w.mz[src];
            vf[q] = w.mf[src];
            vl[q] = w.ml[src];
            fl[q] = ok && (fabs(rho * vz[q]) > tol);
            bal[q] = __ballot_sync(0xffffffffu, fl[q]);
            wcnt += __popc(bal[q]);
        }
        int tot;
        const int wpre = defl_warp_prefix<T>(wcnt, iscan, &tot);
        int before = wpre;
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            const int idx = wbase + 32 * q + lane;
            if (idx < r1) {
                const int na = before + __popc(bal[q] & lt); // survivors before this row
                if (fl[q]) {
                    const long long o = gs + carry_a + na;
                    w.ad[o] = vd[q];
                    w.az[o] = vz[q];
                    w.af[o] = vf[q];
                    w.al[o] = vl[q];
                    w.amap[o] = idx;
                    w.gmark[o] = 0;
                } else {
                    const long long o = gs + carry_z + (idx - base) - na;
                    w.zd[o] = vd[q];
                    w.zf[o] = vf[q];
                    w.zl[o] = vl[q];
                    w.zmap[o] = idx;
                }
            }
            before += __popc(bal[q]);
        }
        const int valid = (r1 - base) < EPT * T ? (r1 - base) : EPT * T;
        carry_a += tot;
        carry_z += valid - tot;
    }
    return carry_a;
}

// Close-pole clusters whose run starts at an active index in [i0, i1): one
// thread walks each run of gaps <= tol (it may read and rotate entries past
// i1; no other thread touches them).  Returns whether this thread rotated
// any entry out.
template <int T>
__device__ bool defl_close_walk(const Ws &w, long long gs, int Kz, double tol, int i0, int i1) {
    bool rotated = false;
    for (int i = i0 + threadIdx.x; i < i1; i += T) {
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
            w.gr[gs + x] = r;
            w.gbase[gs + x] = base;
            rotated = true;
            ++x;
        }
        w.az[gs + base] = zb;
        w.af[gs + base] = fb;
        w.al[gs + base] = lb;
    }
    return rotated;
}

// Active entries [r0, r1) that remain poles (not rotated out).
template <int T>
__device__ int defl_count_poles(const Ws &w, long long gs, int r0, int r1, int *iscan) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int wcnt = 0;
    for (int base = r0; base < r1; base += kDeflEPT * T) {
        const int wbase = base + wid * (kDeflEPT * 32);
#pragma unroll
        for (int q = 0; q < kDeflEPT; ++q) {
            const int idx = wbase + 32 * q + lane;
            const bool f = idx < r1 && w.gmark[gs + idx] == 0;
            wcnt += __popc(__ballot_sync(0xffffffffu, f));
        }
    }
    int tot;
    defl_warp_prefix<T>(wcnt, iscan, &tot);
    return tot;
}

// Compaction 2 of active entries [r0, r1): poles to the padded pole slice
// from carry_p, rotated-out members to their list from carry_g.  Returns
// this thread's part of sum z^2 over the poles it moved; *end_p gets
// carry_p plus the poles.
template <int T>
__device__ double defl_compact_poles(const Ws &w, long long gs, long long po, int r0, int r1,
                                     int carry_p, int carry_g, int *iscan, int *end_p) {
    constexpr int EPT = kDeflEPT;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    double zn = 0.0;
    for (int base = r0; base < r1; base += EPT * T) {
        const int wbase = base + wid * (EPT * 32);
        bool fl[EPT];
        unsigned bal[EPT];
        double vd[EPT], vz[EPT], vf[EPT], vl[EPT];
        int wcnt = 0;
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            const int idx = wbase + 32 * q + lane;
            const bool ok = idx < r1;
            const long long src = gs + (ok ? idx : r0);
            vd[q] = w.ad[src];
            vz[q] = w.az[src];
            vf[q] = w.af[src];
            vl[q] = w.al[src];
            fl[q] = ok && (w.gmark[src] == 0);
            bal[q] = __ballot_sync(0xffffffffu, fl[q]);
            wcnt += __popc(bal[q]);
        }
        int tot;
        const int wpre = defl_warp_prefix<T>(wcnt, iscan, &tot);
        int before = wpre;
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            const int idx = wbase + 32 * q + lane;
            if (idx < r1) {
                const int np = before + __popc(bal[q] & lt); // poles before this entry
                if (fl[q]) {
                    const long long o = po + carry_p + np;
                    w.pd[o] = vd[q];
                    w.pz[o] = vz[q];
                    w.pf[o] = vf[q];
                    w.pl[o] = vl[q];
                    w.pmap[o] = idx;
                    zn += vz[q] * vz[q];
                } else {
                    const long long o = gs + carry_g + (idx - base) - np;
                    w.gd[o] = vd[q];
                    w.gf[o] = vf[q];
                    w.gl[o] = vl[q];
                    w.gpos[o] = idx;
                }
            }
            before += __popc(bal[q]);
        }
        const int valid = (r1 - base) < EPT * T ? (r1 - base) : EPT * T;
        carry_p += tot;
        carry_g += valid - tot;
    }
    *end_p = carry_p;
    return zn;
}

// Deflation tolerance inputs of node g: rho, max|d| from the ends of the two
// sorted child spectra.
__device__ inline void defl_node_scalars(const KArgs &a, const NodeGeom &G, double *rho,
                                         double *maxd) {
    const Ws &w = a.w;
    const long long gs = G.gstart;
    const double *Ad = w.cd + gs;
    const double *Bd = w.cd + gs + G.m1;
    const int m2 = G.m - G.m1;
    *rho = 2.0 * inst_scale(w, G.inst) * fabs(a.E[gs + G.m1 - 1]);
    *maxd = fmax(fmax(fabs(Ad[0]), fabs(Ad[G.m1 - 1])), fmax(fabs(Bd[0]), fabs(Bd[m2 - 1])));
}

// Node scalars, then the level plan by the last CTA to finish (unless the
// level runs k_plan).
template <int T>
__device__ void defl_finish(const KArgs &a, int g, int K, int Kz, double rho, double tol,
                            double zn, bool writer, double *red, int *iscan, int *s_last) {
    const Ws &w = a.w;
    if (writer && threadIdx.x == 0) {
        w.nK[g] = K;
        w.nKz[g] = Kz;
        w.nrho[g] = rho;
        w.ntol[g] = tol;
        w.nzn[g] = zn;
    }
    if (!a.plan_inline) {
        return;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const int t = atomicAdd(&w.hdr->lvl[a.k].ticket, 1);
        *s_last = (t == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (!*s_last) {
        return;
    }
    __threadfence();
    level_plan<T>(a, red, iscan);
}

// One CTA per merge node.
template <int T>
__global__ void __launch_bounds__(T) k_merge_deflate(KArgs a) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    __shared__ double red[32];
    __shared__ int iscan[32];
    __shared__ int s_last;
    const int g = blockIdx.x;
    const NodeGeom G = node_geom(a.F, a.k, g);
    const Ws &w = a.w;
    const long long gs = G.gstart;
    const int m = G.m;
    double rho, maxd;
    defl_node_scalars(a, G, &rho, &maxd);
    double lz = 0.0;
    for (int e = threadIdx.x; e < m; e += T) {
        lz = fmax(lz, fabs(w.mz[gs + e]));
    }
    const double maxz = block_max<T>(lz, red);
    const double tol = kDeflTolScale * DBL_EPSILON * fmax(maxd, maxz);

    const int Kz = defl_compact_active<T>(w, gs, 0, m, rho, tol, 0, 0, iscan);
    __syncthreads();
    defl_close_walk<T>(w, gs, Kz, tol, 0, Kz);
    __syncthreads();
    int K;
    double zn = defl_compact_poles<T>(w, gs, G.poff, 0, Kz, 0, 0, iscan, &K);
    zn = block_sum<T>(zn, red);
    defl_finish<T>(a, g, K, Kz, rho, tol, zn, true, red, iscan, &s_last);
}

// A cluster of C CTAs per merge node (the large merges near the top of the
// tree, which one CTA would stream alone).  CTA r of the cluster owns rows
// [r S, (r+1) S) of the node (S a whole number of chunks), then the same
// share of the active list.  The tolerance maximum and the compaction counts
// are exchanged through distributed shared memory between cluster barriers,
// so each CTA scatters from its exact offset and the lists come out exactly
// as the one-CTA kernel writes them (only sum z^2 is added in another
// order).  The close-pole walk reads the whole active list from global
// memory after a cluster barrier.
template <int T>
__global__ void __launch_bounds__(T) k_merge_deflate_cl(KArgs a) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    namespace cg = cooperative_groups;
    __shared__ double red[32];
    __shared__ int iscan[32];
    __shared__ int s_last;
    __shared__ double s_val;
    __shared__ int s_cnt;
    __shared__ int s_rot;
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks();
    const int rank = (int)cl.block_rank();
    const int g = blockIdx.x / C;
    const NodeGeom G = node_geom(a.F, a.k, g);
    const Ws &w = a.w;
    const long long gs = G.gstart;
    const int m = G.m;
    constexpr int chunk = kDeflEPT * T;
    double rho, maxd;
    defl_node_scalars(a, G, &rho, &maxd);

    const int S = ((m + C - 1) / C + chunk - 1) / chunk * chunk;
    const int r0 = min(m, rank * S), r1 = min(m, r0 + S);
    double lz = 0.0;
    for (int e = r0 + threadIdx.x; e < r1; e += T) {
        lz = fmax(lz, fabs(w.mz[gs + e]));
    }
    lz = block_max<T>(lz, red);
    if (threadIdx.x == 0) {
        s_val = lz;
    }
    cl.sync();
    double maxz = 0.0;
    for (int r = 0; r < C; ++r) {
        maxz = fmax(maxz, *cl.map_shared_rank(&s_val, r));
    }
    const double tol = kDeflTolScale * DBL_EPSILON * fmax(maxd, maxz);

    // compaction 1
    const int na = defl_count_active<T>(w, gs, r0, r1, rho, tol, iscan);
    if (threadIdx.x == 0) {
        s_cnt = na;
    }
    cl.sync();
    int off_a = 0, Kz = 0;
    for (int r = 0; r < C; ++r) {
        const int c = *cl.map_shared_rank(&s_cnt, r);
        off_a += r < rank ? c : 0;
        Kz += c;
    }
    // the cluster barrier releases and acquires at cluster scope, which
    // orders these global writes for the peer CTAs without a device fence
    defl_compact_active<T>(w, gs, r0, r1, rho, tol, off_a, r0 - off_a, iscan);
    cl.sync();

    // close-pole walk over this CTA's share of chain starts
    const int A = (Kz + C - 1) / C;
    const int rot = __syncthreads_or(
        defl_close_walk<T>(w, gs, Kz, tol, min(Kz, rank * A), min(Kz, rank * A + A)));
    if (threadIdx.x == 0) {
        s_rot = rot;
    }
    cl.sync();
    bool any_rot = false;
    for (int r = 0; r < C; ++r) {
        any_rot |= *cl.map_shared_rank(&s_rot, r) != 0;
    }

    // compaction 2 (with nothing rotated out, every active entry is a pole
    // and no count is needed)
    const int S2 = ((Kz + C - 1) / C + chunk - 1) / chunk * chunk;
    const int q0 = min(Kz, rank * S2), q1 = min(Kz, q0 + S2);
    int off_p = q0, K = Kz;
    if (any_rot) {
        const int np = defl_count_poles<T>(w, gs, q0, q1, iscan);
        if (threadIdx.x == 0) {
            s_cnt = np;
        }
        cl.sync();
        off_p = 0;
        K = 0;
        for (int r = 0; r < C; ++r) {
            const int c = *cl.map_shared_rank(&s_cnt, r);
            off_p += r < rank ? c : 0;
            K += c;
        }
    }
    int end_p;
    double zn = defl_compact_poles<T>(w, gs, G.poff, q0, q1, off_p, q0 - off_p, iscan, &end_p);
    zn = block_sum<T>(zn, red);
    if (threadIdx.x == 0) {
        s_val = zn;
    }
    cl.sync();
    double zt = 0.0;
    if (rank == 0) {
        for (int r = 0; r < C; ++r) {
            zt += *cl.map_shared_rank(&s_val, r);
        }
    }
    // no CTA leaves while a peer may still read its shared memory
    cl.sync();
    defl_finish<T>(a, g, K, Kz, rho, tol, zt, rank == 0, red, iscan, &s_last);
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
    unsigned pend;               // stages with a copy issued and not yet waited for
    unsigned long long wait_ns;  // bound of one tile wait
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
    ts.pend |= 1u << stage;
}

// Wait for the copies of one stage, every thread of the block; true when
// they landed within the wait limit for all threads.  On a timeout the
// stage stays pending (tiles_drain waits for it) and the phase unchanged.
template <int NA>
__device__ inline bool tiles_wait(TileSet<NA> &ts, int stage) {
    const bool ok = mbar_wait(&ts.bar[stage], ts.phase[stage], ts.wait_ns);
    if (!__syncthreads_and(ok)) {
        return false;
    }
    ts.phase[stage] ^= 1u;
    ts.pend &= ~(1u << stage);
    return true;
}

// After a timeout: wait (bounded by kDrainWaitNs) for the copies still in
// flight into this block's shared memory, so none lands after the block
// has moved on or exited.
template <int NA>
__device__ inline void tiles_drain(TileSet<NA> &ts) {
#pragma unroll
    for (int st = 0; st < 2; ++st) {
        if (ts.pend & (1u << st)) {
            mbar_wait(&ts.bar[st], ts.phase[st], kDrainWaitNs);
            ts.phase[st] ^= 1u;
        }
    }
    ts.pend = 0u;
    __syncthreads();
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
            if (!tiles_wait(ts, 0)) {
                return false;
            }
            if (ts.ntiles > 1 && !tiles_wait(ts, 1)) {
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
        if (!tiles_wait(ts, st)) {
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
                                   int count, unsigned long long wait_ns) {
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
    ts.pend = 0u;
    ts.wait_ns = wait_ns;
}

__device__ inline void record_error(WsHeader *h, int code) {
    atomicCAS(&h->status, 0, code);
}

// Item -> node lookup (table written by the level plan).
__device__ inline int item_node(const int *table, int item) {
    __syncthreads();
    return table[item];
}

// Per-root / per-pole work of the three sweep phases, shared by the two
// roles.  The warp role reads poles through L1 (__ldg); the CTA role reads
// them from shared-memory tiles.

struct RootIO {
    const Ws *w;
    long long po;
    int K;
};

__device__ inline void secular_store(const Ws &w, const KArgs &a, long long po,
                                     int r, const SecRoot &st) {
    const long long o = po + r;
    w.rorg[o] = st.org;
    w.rdo[o] = st.dorg;
    w.rtau[o] = st.tau;
    w.rlam[o] = st.dorg + st.tau;
}

// Iteration counters of the level diagnostics, reduced over the warp first:
// one atomic per warp instead of one per root keeps the same-address
// traffic at L2 off the critical path.  Called by every lane of the warp;
// `mine` marks the lanes that report a root.
__device__ inline void secular_diag_warp(const Ws &w, int k, bool mine, const SecRoot &st) {
    const unsigned full = 0xffffffffu;
    const int it = mine ? st.iter : 0;
    const int fl = mine ? st.failed : 0;
    const int sum = __reduce_add_sync(full, it);
    const int mx = __reduce_max_sync(full, it);
    const int nf = __reduce_add_sync(full, fl);
    if ((threadIdx.x & 31) == 0) {
        brdc_level_diagnostics *dg = &w.hdr->diag[k];
        if (sum != 0) {
            atomicAdd(&dg->secular_iter_sum, sum);
            atomicMax(&dg->secular_iter_max, mx);
        }
        if (nf != 0) {
            atomicAdd(&dg->secular_iter_failed, nf);
            atomicAdd(&w.hdr->nonconv, nf);
        }
    }
}

__device__ inline void secular_single(const Ws &w, long long po, double rho) {
    const double z0 = w.pz[po];
    const double t = rho * z0 * z0;
    w.rorg[po] = 0;
    w.rdo[po] = w.pd[po];
    w.rtau[po] = t;
    w.rlam[po] = w.pd[po] + t;
}

// Sums of one root over poles [j0, j0+cnt) taken with stride tpr from lane
// l, for a block of roots whose bracket poles p all lie in [pmin, r1-1].  The
// span is cut into three contiguous segments -- poles left of every root's
// bracket, the few around the brackets, poles right of every bracket -- so
// the outer two run as branch-free unrolled loops.  Each accumulator still
// receives its poles in increasing order, as in a single pass.
__device__ inline int seg_first(int x, int l, int tpr) {
    // smallest jj >= x with jj % tpr == l (x >= 0, tpr a power of two)
    return x + ((l - x) & (tpr - 1));
}

template <typename LD>
__device__ inline void secular_span(SecSums &sum, const SecRoot &st, int j0,
                                    int cnt, int l, int tpr, int pmin, int r1,
                                    LD ld) {
    int lo_end = pmin - j0;
    lo_end = lo_end < 0 ? 0 : (lo_end > cnt ? cnt : lo_end);
    int mid_end = r1 + 1 - j0;
    mid_end = mid_end < 0 ? 0 : (mid_end > cnt ? cnt : mid_end);
#pragma unroll 4
    for (int jj = l; jj < lo_end; jj += tpr) {
        double dj, zj;
        ld(jj, &dj, &zj);
        sec_accum_left(sum, st, dj, zj);
    }
    for (int jj = seg_first(lo_end, l, tpr); jj < mid_end; jj += tpr) {
        double dj, zj;
        ld(jj, &dj, &zj);
        sec_accum(sum, st, j0 + jj, dj, zj);
    }
#pragma unroll 4
    for (int jj = seg_first(mid_end, l, tpr); jj < cnt; jj += tpr) {
        double dj, zj;
        ld(jj, &dj, &zj);
        sec_accum_right(sum, st, dj, zj);
    }
}

__device__ inline void sums_reduce(SecSums &sum, int tpr) {
    for (int o = tpr >> 1; o > 0; o >>= 1) {
        SecSums other;
        other.psi = __shfl_xor_sync(0xffffffffu, sum.psi, o);
        other.dpsi = __shfl_xor_sync(0xffffffffu, sum.dpsi, o);
        other.phi = __shfl_xor_sync(0xffffffffu, sum.phi, o);
        other.dphi = __shfl_xor_sync(0xffffffffu, sum.dphi, o);
        other.err = __shfl_xor_sync(0xffffffffu, sum.err, o);
        sec_combine(sum, other);
    }
}

__device__ inline double group_sum(double v, int tpr) {
    for (int o = tpr >> 1; o > 0; o >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}

__device__ inline double group_prod(double v, int tpr) {
    for (int o = tpr >> 1; o > 0; o >>= 1) {
        v *= __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}

__device__ inline double lowner_value(const Ws &w, long long po, int i,
                                      double prod, double rho) {
    const double zi = w.pz[po + i];
    const double mag = sqrt(fmax(-prod, 0.0));
    double wi = zi < 0.0 ? -mag : mag;
    if (!(mag > 0.0) || !isfinite(mag)) {
        wi = zi * sqrt(rho);
    }
    return wi;
}

__device__ inline int block_role_setup(uint64_t *bars) {
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    return 0;
}

// ---------------------------------------------------------------- roots
// Blocks [0, cta_blocks) serve the CTA-role merges, the others the warp-role
// merges (8 warps per block, each on its own work item).
constexpr int kWarpsPerBlock = kSweepThreads / 32;

// The phases below are device functions over the grid's two roles, run back
// to back by k_sweeps.  CTA-role blocks set up their two mbarriers once (ph
// holds their phase bits across phases).  Each returns false after a barrier
// timeout (recorded in the workspace status).
__device__ bool sweep_secular(const KArgs &a, int cta_blocks, double *smem, uint64_t *bars,
                              unsigned *ph) {
    const Ws &w = a.w;
    const LevelCtl *ctl = &w.hdr->lvl[a.k];
    const double eps = DBL_EPSILON;
    const int max_iter = w.hdr->max_iter;

    if ((int)blockIdx.x >= cta_blocks) {
        const int tpr = ctl->tpr_w;
        const int Rw = 32 / tpr;
        const int items = ctl->items_w;
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int grp = lane / tpr, l = lane % tpr;
        const int stride = ((int)gridDim.x - cta_blocks) * kWarpsPerBlock;
        for (int item = ((int)blockIdx.x - cta_blocks) * kWarpsPerBlock + warp;
             item < items; item += stride) {
            const int g = w.items_w[item];
            const NodeGeom G = node_geom(a.F, a.k, g);
            const int K = w.nK[g];
            const double rho = w.nrho[g];
            const long long po = G.poff;
            if (K == 1) {
                if (lane == 0) {
                    secular_single(w, po, rho);
                }
                continue;
            }
            const int r0 = (item - w.pref_w[g]) * Rw;
            const int r1 = (r0 + Rw < K) ? r0 + Rw : K;
            const int pmin = (r0 < K - 2) ? r0 : K - 2;
            const int r = r0 + grp;
            const bool active = r < K;
            const double *pd = w.pd + po;
            const double *pz = w.pz + po;
            SecRoot st;
            if (active) {
                sec_init(st, r, K, pd, pz, rho, w.nzn[g]);
            } else {
                st.stage = 2;
            }
            for (;;) {
                SecSums sum;
                sec_zero(sum);
                if (active && st.stage != 2) {
                    secular_span(sum, st, 0, K, l, tpr, pmin, r1,
                                 [&](int j, double *dj, double *zj) {
                                     *dj = __ldg(pd + j);
                                     *zj = __ldg(pz + j);
                                 });
                }
                sums_reduce(sum, tpr);
                if (active && st.stage != 2) {
                    sec_after_sweep(st, sum, eps, max_iter);
                }
                if (__all_sync(0xffffffffu, (!active) || st.stage == 2)) {
                    break;
                }
            }
            if (active && l == 0) {
                secular_store(w, a, po, r, st);
            }
            secular_diag_warp(w, a.k, active && l == 0, st);
        }
        return true;
    }

    // CTA role.  A block serves one merge at a time from shared-memory pole
    // tiles; each warp iterates a run of Rw consecutive roots (lane group grp
    // on root run + grp) and, once every root of its run has converged,
    // takes the next run at the following sweep boundary.  Runs come from the
    // block's current item (R consecutive roots), items from the level's
    // counter, so lanes stay busy until the level's pool is empty instead of
    // each item sweeping as long as its slowest root, and the blocks balance
    // themselves.  A root's arithmetic does not depend on when or where it
    // runs: its window [pmin, r1] is fixed by its run.
    const int tpr = ctl->tpr_c;
    const int R = kSweepThreads / tpr;
    const int Rw = 32 / tpr;
    const int runs = R / Rw; // runs per item (= warps per block)
    const int items = ctl->items_c;
    const int warp = threadIdx.x >> 5;
    const int grp = (threadIdx.x & 31) / tpr, lane = threadIdx.x % tpr;
    __shared__ int s_item;            // item the runs come from (-1: none)
    __shared__ int s_next;            // next run of s_item
    __shared__ int s_pending;         // fetched item of the next merge (-1: none yet)
    __shared__ int s_run[kWarpsPerBlock];
    if (threadIdx.x == 0) {
        s_pending = atomicAdd(&w.hdr->lvl[a.k].citem, 1);
    }
    __syncthreads();
    for (;;) {
        const int first = s_pending;
        if (first >= items) {
            break;
        }
        const int g = w.items_c[first];
        const NodeGeom G = node_geom(a.F, a.k, g);
        const int K = w.nK[g];
        const double rho = w.nrho[g];
        const long long po = G.poff;
        const int item0 = w.pref_c[g], item1 = w.pref_c[g + 1];
        __syncthreads();
        if (threadIdx.x == 0) {
            s_item = first;
            s_next = 0;
            s_pending = -1;
        }
        TileSet<2> ts;
        const double *srcs[2] = {w.pd, w.pz};
        tiles_setup<2>(ts, smem, bars, srcs, po, K, w.hdr->wait_ns);
        ts.phase[0] = ph[0];
        ts.phase[1] = ph[1];
        SecRoot st;
        st.stage = 2;
        bool wlive = false; // this warp has a run (warp-uniform)
        bool active = false;
        int r = 0, pmin = 0, r1 = 0;
        bool ok = true;
        for (;;) {
            // sweep boundary: runs for the warps without one (-1 asks, -2
            // keeps the current run)
            if ((threadIdx.x & 31) == 0) {
                s_run[warp] = wlive ? -2 : -1;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                for (int q = 0; q < kWarpsPerBlock; ++q) {
                    if (s_run[q] != -1) {
                        continue;
                    }
                    while (s_item >= 0) {
                        if (s_next < runs) {
                            const int root0 = (s_item - item0) * R + s_next * Rw;
                            ++s_next;
                            if (root0 < K) {
                                s_run[q] = root0;
                                break;
                            }
                            s_next = runs; // the merge's last, partial item
                            continue;
                        }
                        const int it = atomicAdd(&w.hdr->lvl[a.k].citem, 1);
                        if (it >= item0 && it < item1) {
                            s_item = it;
                            s_next = 0;
                        } else {
                            s_pending = it;
                            s_item = -1;
                        }
                    }
                }
            }
            __syncthreads();
            const int run = s_run[warp];
            if (!wlive && run >= 0) {
                r = run + grp;
                active = r < K;
                pmin = (run < K - 2) ? run : K - 2;
                r1 = (run + Rw < K) ? run + Rw : K;
                if (active) {
                    sec_init(st, r, K, w.pd + po, w.pz + po, rho, w.nzn[g]);
                } else {
                    st.stage = 2;
                }
                wlive = true;
            }
            if (!__syncthreads_or(wlive)) {
                break; // the merge is done
            }
            SecSums sum;
            sec_zero(sum);
            const bool live = wlive && active && st.stage != 2;
            ok = tiles_sweep<2>(ts, [&](int j0, int cnt, double *const *b) {
                if (live) {
                    const double *bd = b[0];
                    const double *bz = b[1];
                    secular_span(sum, st, j0, cnt, lane, tpr, pmin, r1,
                                 [&](int jj, double *dj, double *zj) {
                                     *dj = bd[jj];
                                     *zj = bz[jj];
                                 });
                }
            });
            if (!ok) {
                break;
            }
            if (wlive) {
                sums_reduce(sum, tpr);
                if (live) {
                    sec_after_sweep(st, sum, eps, max_iter);
                }
                if (__all_sync(0xffffffffu, (!active) || st.stage == 2)) {
                    if (active && lane == 0) {
                        secular_store(w, a, po, r, st);
                    }
                    secular_diag_warp(w, a.k, active && lane == 0, st);
                    wlive = false;
                    active = false;
                }
            }
        }
        ph[0] = ts.phase[0];
        ph[1] = ts.phase[1];
        if (!ok) {
            tiles_drain(ts);
            record_error(w.hdr, kErrBarrierTimeout);
            return false;
        }
        __syncthreads();
        if (threadIdx.x == 0 && s_pending < 0) {
            s_pending = atomicAdd(&w.hdr->lvl[a.k].citem, 1);
        }
        __syncthreads();
    }
    return true;
}


// ------------------------------------------------------------- Loewner z
// For every pole i:  w_i = sign(z_i) * sqrt(-prod_j delta_i(j) /
// prod_{j != i} (d_i - d_j)),  delta_i(j) = (d_i - d_org(j)) - tau_j: the
// recomputation of cpu/src/dlaed9_br.f:181-266 (WPROD), one lane group per
// pole sweeping the roots.  Instance roots are skipped (no parent reads
// their rows).
// (rdo and rtau are read through L2: k_sweeps writes them in the same launch.)
__device__ bool sweep_lowner(const KArgs &a, int cta_blocks, double *smem, uint64_t *bars,
                             unsigned *ph) {
    const Ws &w = a.w;
    const LevelCtl *ctl = &w.hdr->lvl[a.k];

    if ((int)blockIdx.x >= cta_blocks) {
        const int tpr = ctl->tpr_w;
        const int Rw = 32 / tpr;
        const int items = ctl->items_w;
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int grp = lane / tpr, l = lane % tpr;
        const int stride = ((int)gridDim.x - cta_blocks) * kWarpsPerBlock;
        for (int item = ((int)blockIdx.x - cta_blocks) * kWarpsPerBlock + warp;
             item < items; item += stride) {
            const int g = w.items_w[item];
            const NodeGeom G = node_geom(a.F, a.k, g);
            if (G.depth == 0) {
                continue;
            }
            const int K = w.nK[g];
            const long long po = G.poff;
            const int i = (item - w.pref_w[g]) * Rw + grp;
            const bool active = i < K;
            // two factors per step share one reciprocal (lowner_pair)
            double prod = 1.0;
            if (active) {
                const double di = w.pd[po + i];
                const double *rdo = w.rdo + po;
                const double *rtau = w.rtau + po;
                const double *pd = w.pd + po;
                int j = l;
#pragma unroll 2
                for (; j + tpr < K; j += 2 * tpr) {
                    const int j2 = j + tpr;
                    const double dl = (di - __ldcg(rdo + j)) - __ldcg(rtau + j);
                    const double dl2 = (di - __ldcg(rdo + j2)) - __ldcg(rtau + j2);
                    prod *= lowner_pair(dl, j == i ? 1.0 : di - __ldg(pd + j), dl2,
                                        j2 == i ? 1.0 : di - __ldg(pd + j2));
                }
                if (j < K) {
                    const double dl = (di - __ldcg(rdo + j)) - __ldcg(rtau + j);
                    prod *= dl * brdc_rcp(j == i ? 1.0 : di - __ldg(pd + j));
                }
            }
            prod = group_prod(prod, tpr);
            if (active && l == 0) {
                w.pw[po + i] = lowner_value(w, po, i, prod, w.nrho[g]);
            }
        }
        return true;
    }

    const int tpr = ctl->tpr_c;
    const int R = kSweepThreads / tpr;
    const int items = ctl->items_c;
    const int grp = threadIdx.x / tpr, lane = threadIdx.x % tpr;
    for (int item = blockIdx.x; item < items; item += cta_blocks) {
        const int g = item_node(w.items_c, item);
        const NodeGeom G = node_geom(a.F, a.k, g);
        if (G.depth == 0) {
            continue;
        }
        const int K = w.nK[g];
        const long long po = G.poff;
        const int i = (item - w.pref_c[g]) * R + grp;
        const bool active = i < K;
        const double di = active ? w.pd[po + i] : 0.0;
        double prod = 1.0;
        TileSet<3> ts;
        const double *srcs[3] = {w.rdo, w.rtau, w.pd};
        tiles_setup<3>(ts, smem, bars, srcs, po, K, w.hdr->wait_ns);
        ts.phase[0] = ph[0];
        ts.phase[1] = ph[1];
        const bool ok = tiles_sweep<3>(ts, [&](int j0, int cnt, double *const *b) {
            if (active) {
                int jj = lane;
                // unrolled so that the next pair's shared-memory loads issue
                // under this pair's product (Toeplitz 65,536: 21.03 ->
                // 20.75 ms with the rows loop below, the same bits)
#pragma unroll 4
                for (; jj + tpr < cnt; jj += 2 * tpr) {
                    const int j = j0 + jj, jj2 = jj + tpr;
                    const double dl = (di - b[0][jj]) - b[1][jj];
                    const double dl2 = (di - b[0][jj2]) - b[1][jj2];
                    prod *= lowner_pair(dl, j == i ? 1.0 : di - b[2][jj], dl2,
                                        j + tpr == i ? 1.0 : di - b[2][jj2]);
                }
                if (jj < cnt) {
                    const double dl = (di - b[0][jj]) - b[1][jj];
                    prod *= dl * brdc_rcp(j0 + jj == i ? 1.0 : di - b[2][jj]);
                }
            }
        });
        ph[0] = ts.phase[0];
        ph[1] = ts.phase[1];
        if (!ok) {
            tiles_drain(ts);
            record_error(w.hdr, kErrBarrierTimeout);
            return false;
        }
        prod = group_prod(prod, tpr);
        if (active && lane == 0) {
            w.pw[po + i] = lowner_value(w, po, i, prod, w.nrho[g]);
        }
        __syncthreads();
    }
    return true;
}


// ----------------------------------------------------------- boundary rows
// Root s: u_i = w_i / delta_i(s), normalised; new first row = sum_i f_i u_i,
// new last row = sum_i l_i u_i: the streamed update of
// cpu/src/dlaed9_br.f:272-334 with the compact delta.  Written to rf/rl;
// k_place puts them in order.
// (rdo, rtau and pw are read through L2: k_sweeps writes them in the same
// launch.)
__device__ bool sweep_rows(const KArgs &a, int cta_blocks, double *smem, uint64_t *bars,
                           unsigned *ph) {
    const Ws &w = a.w;
    const LevelCtl *ctl = &w.hdr->lvl[a.k];

    if ((int)blockIdx.x >= cta_blocks) {
        const int tpr = ctl->tpr_w;
        const int Rw = 32 / tpr;
        const int items = ctl->items_w;
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int grp = lane / tpr, l = lane % tpr;
        const int stride = ((int)gridDim.x - cta_blocks) * kWarpsPerBlock;
        for (int item = ((int)blockIdx.x - cta_blocks) * kWarpsPerBlock + warp;
             item < items; item += stride) {
            const int g = w.items_w[item];
            const NodeGeom G = node_geom(a.F, a.k, g);
            if (G.depth == 0) {
                continue;
            }
            const int K = w.nK[g];
            const long long po = G.poff;
            const int s = (item - w.pref_w[g]) * Rw + grp;
            const bool root = s < K;
            double a1 = 0.0, a2 = 0.0, s2 = 0.0;
            if (root) {
                const double dorg = __ldcg(w.rdo + po + s);
                const double tau = __ldcg(w.rtau + po + s);
                const double *pd = w.pd + po;
                const double *pw = w.pw + po;
                const double *pf = w.pf + po;
                const double *pl = w.pl + po;
                int i = l;
#pragma unroll 2
                for (; i + tpr < K; i += 2 * tpr) {
                    const int i2 = i + tpr;
                    double u, u2;
                    row_pair(__ldcg(pw + i), (__ldg(pd + i) - dorg) - tau, __ldcg(pw + i2),
                             (__ldg(pd + i2) - dorg) - tau, &u, &u2);
                    s2 += u * u;
                    a1 += __ldg(pf + i) * u;
                    a2 += __ldg(pl + i) * u;
                    s2 += u2 * u2;
                    a1 += __ldg(pf + i2) * u2;
                    a2 += __ldg(pl + i2) * u2;
                }
                if (i < K) {
                    const double dl = (__ldg(pd + i) - dorg) - tau;
                    const double u = (dl != 0.0) ? __ldcg(pw + i) * brdc_rcp(dl) : 0.0;
                    s2 += u * u;
                    a1 += __ldg(pf + i) * u;
                    a2 += __ldg(pl + i) * u;
                }
            }
            s2 = group_sum(s2, tpr);
            a1 = group_sum(a1, tpr);
            a2 = group_sum(a2, tpr);
            if (root && l == 0) {
                const double nrm = sqrt(s2);
                w.rf[po + s] = nrm > 0.0 ? a1 / nrm : 0.0;
                w.rl[po + s] = nrm > 0.0 ? a2 / nrm : 0.0;
            }
        }
        return true;
    }

    const int tpr = ctl->tpr_c;
    const int R = kSweepThreads / tpr;
    const int items = ctl->items_c;
    const int grp = threadIdx.x / tpr, lane = threadIdx.x % tpr;
    for (int item = blockIdx.x; item < items; item += cta_blocks) {
        const int g = item_node(w.items_c, item);
        const NodeGeom G = node_geom(a.F, a.k, g);
        if (G.depth == 0) {
            continue;
        }
        const int K = w.nK[g];
        const long long po = G.poff;
        const int s = (item - w.pref_c[g]) * R + grp;
        const bool root = s < K;
        const double dorg = root ? __ldcg(w.rdo + po + s) : 0.0;
        const double tau = root ? __ldcg(w.rtau + po + s) : 0.0;
        double a1 = 0.0, a2 = 0.0, s2 = 0.0;
        TileSet<4> ts;
        const double *srcs[4] = {w.pd, w.pw, w.pf, w.pl};
        tiles_setup<4>(ts, smem, bars, srcs, po, K, w.hdr->wait_ns);
        ts.phase[0] = ph[0];
        ts.phase[1] = ph[1];
        const bool ok = tiles_sweep<4>(ts, [&](int j0, int cnt, double *const *b) {
            if (root) {
                int jj = lane;
#pragma unroll 4
                for (; jj + tpr < cnt; jj += 2 * tpr) {
                    const int jj2 = jj + tpr;
                    double u, u2;
                    row_pair(b[1][jj], (b[0][jj] - dorg) - tau, b[1][jj2],
                             (b[0][jj2] - dorg) - tau, &u, &u2);
                    s2 += u * u;
                    a1 += b[2][jj] * u;
                    a2 += b[3][jj] * u;
                    s2 += u2 * u2;
                    a1 += b[2][jj2] * u2;
                    a2 += b[3][jj2] * u2;
                }
                if (jj < cnt) {
                    const double dl = (b[0][jj] - dorg) - tau;
                    const double u = (dl != 0.0) ? b[1][jj] * brdc_rcp(dl) : 0.0;
                    s2 += u * u;
                    a1 += b[2][jj] * u;
                    a2 += b[3][jj] * u;
                }
            }
        });
        ph[0] = ts.phase[0];
        ph[1] = ts.phase[1];
        if (!ok) {
            tiles_drain(ts);
            record_error(w.hdr, kErrBarrierTimeout);
            return false;
        }
        s2 = group_sum(s2, tpr);
        a1 = group_sum(a1, tpr);
        a2 = group_sum(a2, tpr);
        if (root && lane == 0) {
            const double nrm = sqrt(s2);
            w.rf[po + s] = nrm > 0.0 ? a1 / nrm : 0.0;
            w.rl[po + s] = nrm > 0.0 ? a2 / nrm : 0.0;
        }
        __syncthreads();
    }
    return true;
}


// --------------------------------------------------------------- placement
// One thread per row of the level: every eigenvalue of a merged node (root,
// small-z deflated, rotated out) goes to its place in the node's ascending
// spectrum by rank among the three sorted lists (ties: roots, then small-z,
// then rotated), with its first and last boundary-row entries; instance
// roots write the final eigenvalues to W.
__device__ void place_rows(const KArgs &a, long long total_n) {
    const Ws &w = a.w;
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < total_n;
         x += (long long)gridDim.x * blockDim.x) {
        int g, m, depth, inst;
        long long gs;
        if (!elem_node(a.F, a.k, x, &g, &gs, &m, &depth, &inst)) {
            continue;
        }
        const long long po = (gs + g + 1) & ~1LL;
        const int s = (int)(x - gs);
        const int K = w.nK[g];
        if (K <= a.big_k && a.big_k > 0) {
            continue; // placed by k_level
        }
        const int Kz = w.nKz[g];
        const int ndz = m - Kz, ndg = Kz - K;
        const bool top = (depth == 0);
        const double *zdl = w.zd + gs;
        const double *gdl = w.gd + gs;
        const double *rl = w.rlam + po;
        double val, fo = 0.0, lo = 0.0;
        int pos;
        if (s < K) {
            val = __ldcg(rl + s);
            pos = s + lower_bound_d(zdl, ndz, val) + lower_bound_d(gdl, ndg, val);
            if (!top) {
                fo = __ldcg(w.rf + po + s);
                lo = __ldcg(w.rl + po + s);
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
            a.W[o] = val * inst_unscale(w, inst);
        } else {
            w.nd[o] = val;
            w.nf[o] = fo;
            w.nl[o] = lo;
        }
    }
}


// ------------------------------------------------------------ k_sweeps
// Grid-wide barrier of a cooperative launch (every block resident), on the
// level's counter pair: arrivals, then a generation bump by the last block.
// The wait is bounded by the handle's wait limit (WsHeader::wait_ns); on
// timeout the status records it and the caller leaves.

__device__ inline bool grid_barrier(WsHeader *h, LevelCtl *c) {
    __syncthreads();
    int ok = 1;
    if (threadIdx.x == 0) {
        volatile unsigned *gen = &c->bar_gen;
        const unsigned g = *gen; // before arriving: the last arrival bumps it
        __threadfence();
        if (atomicAdd(&c->bar_count, 1u) + 1u == gridDim.x) {
            c->bar_count = 0u;
            __threadfence();
            atomicAdd(&c->bar_gen, 1u);
        } else {
            const unsigned long long t0 = globaltimer_ns();
            const unsigned long long limit = h->wait_ns;
            while (*gen == g) {
                __nanosleep(100);
                if (globaltimer_ns() - t0 > limit) {
                    ok = 0;
                    record_error(h, kErrGridBarrierTimeout);
                    break;
                }
            }
        }
        __threadfence();
    }
    return __syncthreads_and(ok) != 0;
}

// Roots, Loewner weights, boundary rows and placement of one level in one
// cooperative launch: the four phases above separated by grid barriers
// instead of kernel boundaries.  After k_level (big_k > 0) it returns at
// once when the level plan has no items: k_level finished every merge.
// The roles split the grid in proportion to their pole-root pairs in the
// plan (all blocks to the role that has items when only one has; `tiles` =
// 0: the launch has no tile memory and every block takes the warp role).  `rows` = 0 skips the
// Loewner and rows phases (every merge an instance root).
__global__ void __launch_bounds__(kSweepThreads)
    k_sweeps(KArgs a, int tiles, int rows, long long total_n) {
    pdl_begin();
    if (halted(a.w.hdr)) {
        return;
    }
    extern __shared__ __align__(16) double smem[];
    __shared__ __align__(8) uint64_t bars[2];
    WsHeader *h = a.w.hdr;
    LevelCtl *ctl = &h->lvl[a.k];
    const int iw = __ldcg(&ctl->items_w), ic = __ldcg(&ctl->items_c);
    if (a.big_k > 0 && iw + ic == 0) {
        return;
    }
    int cta_blocks = 0;
    if (tiles && ic > 0) {
        cta_blocks = (int)gridDim.x;
        if (iw > 0) {
            const double wc = __ldcg(&ctl->work_c), ww = __ldcg(&ctl->work_w);
            const int share = (int)((double)gridDim.x * wc / fmax(wc + ww, 1.0) + 0.5);
            cta_blocks = max(1, min((int)gridDim.x - 1, min(share, ic)));
        }
    }
    unsigned ph[2] = {0u, 0u};
    if ((int)blockIdx.x < cta_blocks) {
        block_role_setup(bars);
    }
    // a block whose tile wait timed out skips its work but keeps to the
    // barriers, so the others do not wait for it
    bool ok = sweep_secular(a, cta_blocks, smem, bars, ph);
    if (!grid_barrier(h, ctl)) {
        return;
    }
    if (rows) {
        if (ok) {
            ok = sweep_lowner(a, cta_blocks, smem, bars, ph);
        }
        if (!grid_barrier(h, ctl)) {
            return;
        }
        if (ok) {
            ok = sweep_rows(a, cta_blocks, smem, bars, ph);
        }
        if (!grid_barrier(h, ctl)) {
            return;
        }
    }
    if (ok) {
        place_rows(a, total_n);
    }
}

// Max-norm max(|D|, |E|) of every instance, as the bits of a non-negative
// double (which order like the integers): grid-wide with one
// atomic per block for a single matrix, one warp per instance for a batch.
// For a single matrix read from host memory (brdc_dstebr_host), cD and cE
// receive the device images of D and E that the rest of the solve reads.
// A NaN or an infinity anywhere in D or E (the ignored E slot at the end
// of each instance excepted) sets kErrNonFinite: nothing after k_norm runs,
// and brdc_get_info reports it.  (fmax would drop a NaN silently.)
__global__ void __launch_bounds__(256) k_norm(Forest F, const double *D, const double *E,
                                              long long *out, WsHeader *h, double *cD,
                                              double *cE) {
    pdl_begin();
    const int lane = threadIdx.x & 31;
    bool bad = false;
    if (F.B == 1) {
        const long long n = F.n0;
        double mx = 0.0;
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
             i += (long long)gridDim.x * blockDim.x) {
            const double dr = D[i];
            if (cD != nullptr) {
                cD[i] = dr;
            }
            const double dv = fabs(dr);
            bad |= !(dv <= DBL_MAX);
            mx = fmax(mx, dv);
            if (i + 1 < n) {
                const double er = E[i];
                if (cE != nullptr) {
                    cE[i] = er;
                }
                const double ev = fabs(er);
                bad |= !(ev <= DBL_MAX);
                mx = fmax(mx, ev);
            }
        }
        __shared__ double red[32];
        mx = block_max<256>(mx, red);
        if (threadIdx.x == 0) {
            atomicMax(out, __double_as_longlong(mx));
        }
        if (bad) {
            record_error(h, kErrNonFinite);
        }
        return;
    }
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long b = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); b < F.B;
         b += warps) {
        const long long lo = F.off[b], hi = F.off[b + 1];
        double mx = 0.0;
        for (long long i = lo + lane; i < hi; i += 32) {
            const double dv = fabs(D[i]);
            bad |= !(dv <= DBL_MAX);
            mx = fmax(mx, dv);
            if (i + 1 < hi) {
                const double ev = fabs(E[i]);
                bad |= !(ev <= DBL_MAX);
                mx = fmax(mx, ev);
            }
        }
        mx = warp_max(mx);
        if (lane == 0) {
            out[b] = __double_as_longlong(mx);
        }
    }
    if (bad) {
        record_error(h, kErrNonFinite);
    }
}

__global__ void k_init(WsHeader *h, int levels, int B, long long total_n,
                       long long leaves, int flags, long long *norm, int max_iter,
                       unsigned long long wait_ns) {
    const int t = threadIdx.x;
    if (t == 0) {
        norm[0] = 0;
    }
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
        h->leaf_sweeps_sum = 0;
        h->max_iter = max_iter;
        h->wait_ns = wait_ns;
    }
    for (int k = t; k < BRDC_MAX_LEVELS; k += blockDim.x) {
        h->lvl[k].ticket = 0;
        h->lvl[k].tpr_w = 1;
        h->lvl[k].tpr_c = 1;
        h->lvl[k].items_w = 0;
        h->lvl[k].items_c = 0;
        h->lvl[k].total_k = 0;
        h->lvl[k].nbig = 0;
        h->lvl[k].bar_count = 0u;
        h->lvl[k].bar_gen = 0u;
        h->lvl[k].citem = 0;
        h->lvl[k].work_w = 0.0;
        h->lvl[k].work_c = 0.0;
        brdc_level_diagnostics z = {};
        z.level = k;
        h->diag[k] = z;
    }
}

} // namespace brdc
