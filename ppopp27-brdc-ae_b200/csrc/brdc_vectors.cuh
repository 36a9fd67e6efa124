// brdc_vectors.cuh -- eigenvectors from a checkpointed BR solve.
//
// The reference's vector path (gpu/src/tridiag_solver.cu:848-1071) carries
// each node's eigenvector matrix up the tree; the values-only solve carries
// only its first and last rows.  Here a checkpointing values solve records
// every merge (merge permutation, deflation lists and Givens chains, poles,
// roots), and the eigenvectors are then assembled bottom-up:
//
//   Q_node = blockdiag(Q_left, Q_right) * M_node
//
// where column t of M_node (m x m, rows in the children's eigenvector
// coordinates) is the node's t-th eigenvector (ascending) in the children's
// eigenbasis:
//   root j:          sum_i u_ij P_i,  u_ij = w_i / delta_ij, normalised,
//                    w the Loewner weights (cpu/src/dlaed9_br.f:181-266),
//                    P_i the active column of pole i after the chains;
//   small-z slot q:  the unit column of its merged position;
//   rotated-out q:   its active column after the chains.
// An active column after the chains is the chain product applied to unit
// columns, which is the chains undone on the rows: the row operations of
// the adjoint's chain reversal.  Rows map to child coordinates through
// amap/zmap (list -> merged position) and morig (merged position -> child
// eigenvalue index).  The two products per node run in k_vec_gemm below, on
// the FP64 tensor cores, each root column written straight to its place.
#pragma once

#include "brdc_kernels.cuh"

namespace brdc {

struct VArgs {
    Forest F;
    Ws w;         // the level's checkpoint slices
    double *M;    // node g's root columns at M + gstart * mstride, column-major, ld m
    long long mstride;
    int k;
    int nodes;
    // eigenvector blocks of the children: the leaves (ld 16) or the level
    // below (node at gstart * child_stride, ld its rows)
    const double *child;
    int leafchild;
    long long child_stride;
    // this level's blocks: node at gstart * out_stride, ld m; the top node
    // at out with ld ldout
    double *out;
    long long out_stride;
    int top;
    long long ldout;
    // the top level writes T's eigenvectors: row i times the sign s_i of
    // T = S |T| S (k_vec_signs)
    const double *sgn;
    // per node and half: the child eigenvector indices (rows of M) that
    // survived the small-z test, in ascending order (k_vec_rows), at
    // rows + gstart + (half ? m1 : 0), and their count at cnt[2 g + half]
    int *rows;
    int *cnt;
};

// Loewner weights of the instance-root merges, which the values solve
// skips (no parent reads their rows): one warp per pole.
__global__ void __launch_bounds__(256) k_vec_lowner(VArgs a) {
    if (halted(a.w.hdr)) {
        return;
    }
    const Ws &w = a.w;
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (int g = 0; g < a.nodes; ++g) {
        const NodeGeom G = node_geom(a.F, a.k, g);
        if (G.depth != 0) {
            continue;
        }
        const int K = w.nK[g];
        const long long po = G.poff;
        for (long long i = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < K;
             i += warps) {
            const double di = w.pd[po + i];
            double prod = 1.0;
            for (int j = lane; j < K; j += 32) {
                const double dl = (di - w.rdo[po + j]) - w.rtau[po + j];
                prod *= dl * brdc_rcp(j == i ? 1.0 : di - w.pd[po + j]);
            }
            for (int o = 16; o > 0; o >>= 1) {
                prod *= __shfl_xor_sync(0xffffffffu, prod, o);
            }
            if (lane == 0) {
                w.pw[po + i] = K == 1 ? w.pz[po + i] * sqrt(w.nrho[g])
                                      : lowner_value(w, po, (int)i, prod, w.nrho[g]);
            }
        }
    }
}

// Row of M (child eigenvector coordinate) of active index a / small-z slot q.
__device__ inline int vec_row_active(const Ws &w, long long gs, int a) {
    return w.morig[gs + w.amap[gs + a]];
}
__device__ inline int vec_row_small(const Ws &w, long long gs, int q) {
    return w.morig[gs + w.zmap[gs + q]];
}

// Position of slot s of a node in its ascending order (the placement rule:
// ties go roots, small-z, rotated-out).
__device__ inline int vec_pos(const Ws &w, long long gs, long long po, int s, int K, int ndz,
                              int ndg) {
    const double *zdl = w.zd + gs;
    const double *gdl = w.gd + gs;
    const double *rl = w.rlam + po;
    if (s < K) {
        return s + lower_bound_d(zdl, ndz, rl[s]) + lower_bound_d(gdl, ndg, rl[s]);
    }
    if (s < K + ndz) {
        const int q = s - K;
        return q + upper_bound_d(rl, K, zdl[q]) + lower_bound_d(gdl, ndg, zdl[q]);
    }
    const int q = s - K - ndz;
    return q + upper_bound_d(rl, K, gdl[q]) + upper_bound_d(zdl, ndz, gdl[q]);
}

// One warp per slot of the level (lanes over rows and poles).  A root s
// writes its column of M at column s (u_i = w_i / delta_i(s) over the
// poles, normalised, then the chains undone on the rows -- chains touch
// disjoint rows, so lanes take different chains); the products turn these
// into the node's root eigenvectors.  A deflated slot is a child
// eigenvector (small-z) or a short rotation combination of some (rotated
// out), written straight to its place in the node's block.  M must be zero.
__global__ void __launch_bounds__(256) k_vec_build(VArgs a, long long total_n) {
    if (halted(a.w.hdr)) {
        return;
    }
    const Ws &w = a.w;
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long x = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); x < total_n;
         x += warps) {
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
        const int m1 = m >> 1;
        if (s < K) {
            double *col = a.M + gs * a.mstride + (long long)s * m;
            const int org = w.rorg[po + s];
            const double dorg = w.rdo[po + s], tau = w.rtau[po + s];
            double s2 = 0.0;
            for (int i = lane; i < K; i += 32) {
                const double dl = (i == org) ? -tau : (w.pd[po + i] - dorg) - tau;
                const double u = w.pw[po + i] / dl;
                s2 += u * u;
            }
            s2 = warp_sum(s2);
            const double inv = 1.0 / sqrt(s2);
            for (int i = lane; i < K; i += 32) {
                const double dl = (i == org) ? -tau : (w.pd[po + i] - dorg) - tau;
                col[vec_row_active(w, gs, w.pmap[po + i])] = w.pw[po + i] / dl * inv;
            }
            __syncwarp();
            // chains: a base has gmark 0 and a member after it
            for (int b0 = lane; b0 + 1 < Kz; b0 += 32) {
                if (w.gmark[gs + b0] != 0 || w.gmark[gs + b0 + 1] == 0) {
                    continue;
                }
                int c = 1;
                while (b0 + c + 1 < Kz && w.gmark[gs + b0 + c + 1] != 0) {
                    ++c;
                }
                const int rb = vec_row_active(w, gs, b0);
                double vb = col[rb];
                for (int kk = c; kk >= 1; --kk) {
                    const long long xg = gs + b0 + kk;
                    const double cc = w.gc[xg], ss = w.gs[xg];
                    const int rx = vec_row_active(w, gs, b0 + kk);
                    // a member is no pole: its row of the column starts at 0
                    const double vx = 0.0;
                    col[rx] = ss * vb + cc * vx;
                    vb = cc * vb - ss * vx;
                }
                col[rb] = vb;
            }
            continue;
        }
        // deflated: a child eigenvector (small-z), or a rotated-out member
        // whose chain, undone on its unit column, leaves c_t at the member
        // (t), s_k * v at the earlier members k and v at the base, v running
        // -s_t, times c_k going down: summed child eigenvectors
        const int pos = vec_pos(w, gs, po, s, K, ndz, ndg);
        double *dst = a.top ? a.out + (long long)pos * a.ldout
                            : a.out + gs * a.out_stride + (long long)pos * m;
        if (s < K + ndz) {
            // small-z deflated: the child eigenvector in its half, zeros in
            // the other, written once (no zero pass and read-back)
            const int e = vec_row_small(w, gs, s - K);
            const bool left = e < m1;
            const int r0 = left ? 0 : m1, r1 = left ? m1 : m;
            const double *c =
                a.leafchild ? a.child + (gs + e) * 16
                            : (left ? a.child + gs * a.child_stride + (long long)e * m1
                                    : a.child + (gs + m1) * a.child_stride +
                                          (long long)(e - m1) * (m - m1));
            for (int r = lane; r < m; r += 32) {
                double v = 0.0;
                if (r >= r0 && r < r1) {
                    v = c[r - r0];
                    v = a.top ? v * a.sgn[r] : v;
                }
                dst[r] = v;
            }
            continue;
        }
        for (int r = lane; r < m; r += 32) {
            dst[r] = 0.0;
        }
        __syncwarp();
        auto add_child = [&](int e, double cf) {
            if (cf == 0.0) {
                return;
            }
            if (e < m1) {
                const double *c = a.leafchild ? a.child + (gs + e) * 16
                                              : a.child + gs * a.child_stride + (long long)e * m1;
                for (int r = lane; r < m1; r += 32) {
                    dst[r] += a.top ? cf * c[r] * a.sgn[r] : cf * c[r];
                }
            } else {
                const int er = e - m1, m2 = m - m1;
                const double *c = a.leafchild
                                      ? a.child + (gs + m1 + er) * 16
                                      : a.child + (gs + m1) * a.child_stride + (long long)er * m2;
                for (int r = lane; r < m2; r += 32) {
                    dst[m1 + r] += a.top ? cf * c[r] * a.sgn[m1 + r] : cf * c[r];
                }
            }
        };
        const int act = w.gpos[gs + (s - K - ndz)];
        int b0 = act;
        while (b0 > 0 && w.gmark[gs + b0] != 0) {
            --b0;
        }
        const int t0 = act - b0;
        add_child(vec_row_active(w, gs, act), w.gc[gs + act]);
        double v = -w.gs[gs + act];
        for (int kk = t0 - 1; kk >= 1; --kk) {
            const long long xg = gs + b0 + kk;
            add_child(vec_row_active(w, gs, b0 + kk), w.gs[xg] * v);
            v *= w.gc[xg];
        }
        add_child(vec_row_active(w, gs, b0), v);
    }
}

// ------------------------------------------------------------ products
// Rows of M that can be nonzero in a root column: the small-z survivors
// (the secular poles and the members rotated into them), as child
// eigenvector indices, split by half and kept in ascending order.  One CTA
// per node.  Every other row of a root column is zero, as LAPACK DLAED3
// uses the deflation (it multiplies only the non-deflated columns of Q).
template <int T>
__global__ void __launch_bounds__(T) k_vec_rows(VArgs a) {
    if (halted(a.w.hdr)) {
        return;
    }
    __shared__ int iscan[32];
    const Ws &w = a.w;
    const int g = blockIdx.x;
    const NodeGeom G = node_geom(a.F, a.k, g);
    const long long gs = G.gstart;
    const int Kz = w.nKz[g];
    int carry_l = 0, carry_r = 0;
    for (int base = 0; base < Kz; base += T) {
        const int i = base + threadIdx.x;
        const int row = i < Kz ? vec_row_active(w, gs, i) : 0;
        const bool right = row >= G.m1;
        int tot;
        const int ex = block_exscan<T>(i < Kz && !right ? 1 : 0, iscan, &tot);
        if (i < Kz) {
            if (!right) {
                a.rows[gs + carry_l + ex] = row;
            } else {
                a.rows[gs + G.m1 + carry_r + (i - base - ex)] = row - G.m1;
            }
        }
        carry_l += tot;
        carry_r += min(T, Kz - base) - tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        a.cnt[2 * g] = carry_l;
        a.cnt[2 * g + 1] = carry_r;
    }
}

// The root eigenvectors of every node of a level, in one launch:
//   Q_node[:, pos(s)] = blockdiag(Q_left, Q_right) * M_node[:, s],  s < K_node,
// as two products per node (top rows with the left child's eigenvector
// block, bottom rows with the right child's), each column written straight
// to its place pos(s) in the node's ascending order (the top level also
// applies the signs of E), so no intermediate product or scatter pass
// exists.  Only the node's own K columns are multiplied, and the inner
// dimension runs over the half's small-z survivors alone (k_vec_rows: the
// only rows of M a root column can have nonzero), gathering those columns
// of the child block and rows of M.  FP64 tensor-core MMA (mma.sync m8n8k4
// .f64, fed from shared memory), 64 x 64 tiles of the output per CTA of
// four warps (32 x 32 each), 16-deep slices of the inner dimension staged
// by cp.async in two buffers.  Grid: x row tiles, y column tiles,
// z = 2 * node + half; tiles past a node's rows or K return at once.
constexpr int kVgBM = 64, kVgBN = 64, kVgBK = 16, kVgPad = 4, kVgThreads = 128;

struct VgSmem {
    // A slice stored k-major (t, r) and B slice (t, s): a warp's fragment
    // loads then touch 16 distinct 8-byte banks per half-warp (row stride
    // 68 doubles = 4 mod 16)
    double A[2][kVgBK][kVgBM + kVgPad];
    double B[2][kVgBK][kVgBN + kVgPad];
    double *dst[kVgBN];
};

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(smem)),
                 "l"(gmem), "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// D = A B + D for one 8x8x4 FP64 tile: lane holds a = A[lane/4][lane%4],
// b = B[lane%4][lane/4], c = D[lane/4][2(lane%4) + {0, 1}].
__device__ __forceinline__ void dmma884(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(kVgThreads) k_vec_gemm(VArgs a) {
    if (halted(a.w.hdr)) {
        return;
    }
    const int g = (int)(blockIdx.z >> 1), half = (int)(blockIdx.z & 1);
    if (g >= a.nodes) {
        return;
    }
    const Ws &w = a.w;
    const NodeGeom G = node_geom(a.F, a.k, g);
    const int K = w.nK[g];
    const int rows = half ? G.m - G.m1 : G.m1;
    const int r0 = (int)blockIdx.x * kVgBM, s0 = (int)blockIdx.y * kVgBN;
    if (r0 >= rows || s0 >= K) {
        return;
    }
    const long long gs = G.gstart;
    const int roff = half ? G.m1 : 0;
    const double *A = a.leafchild ? a.child + (gs + roff) * 16 : a.child + (gs + roff) * a.child_stride;
    const long long lda = a.leafchild ? 16 : rows;
    const double *B = a.M + gs * a.mstride + roff;
    const long long ldb = G.m;
    const int *tl = a.rows + gs + roff;   // inner indices: the half's survivors
    const int nin = a.cnt[2 * g + half];
    __shared__ __align__(16) VgSmem S;
    const int tid = threadIdx.x;
    if (tid < kVgBN) {
        const int s = s0 + tid;
        double *d = nullptr;
        if (s < K) {
            const int Kz = w.nKz[g];
            const int pos = vec_pos(w, gs, G.poff, s, K, G.m - Kz, Kz - K);
            d = a.top ? a.out + (long long)pos * a.ldout + roff
                      : a.out + gs * a.out_stride + (long long)pos * G.m + roff;
        }
        S.dst[tid] = d;
    }
    auto load = [&](int st, int j0) {
#pragma unroll
        for (int q = 0; q < kVgBK * kVgBM / kVgThreads; ++q) {
            const int i = tid + q * kVgThreads;
            const int r = i % kVgBM, j = i / kVgBM;
            const bool v = (r0 + r < rows) && (j0 + j < nin);
            const int t = v ? tl[j0 + j] : 0;
            cp_async8(&S.A[st][j][r], v ? A + (r0 + r) + (long long)t * lda : A, v);
        }
#pragma unroll
        for (int q = 0; q < kVgBK * kVgBN / kVgThreads; ++q) {
            const int i = tid + q * kVgThreads;
            const int j = i % kVgBK, c = i / kVgBK;
            const bool v = (j0 + j < nin) && (s0 + c < K);
            const int t = v ? tl[j0 + j] : 0;
            cp_async8(&S.B[st][j][c], v ? B + t + (long long)(s0 + c) * ldb : B, v);
        }
        cp_async_commit();
    };
    const int lane = tid & 31, wid = tid >> 5;
    const int wr = (wid >> 1) * 32, wc = (wid & 1) * 32;
    const int gid = lane >> 2, tig = lane & 3;
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            acc[i][j][0] = 0.0;
            acc[i][j][1] = 0.0;
        }
    }
    const int nk = (nin + kVgBK - 1) / kVgBK;
    if (nk > 0) {
        load(0, 0);
    }
    __syncthreads(); // S.dst, for an empty inner dimension too
    for (int kt = 0; kt < nk; ++kt) {
        if (kt + 1 < nk) {
            load((kt + 1) & 1, (kt + 1) * kVgBK);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const int st = kt & 1;
#pragma unroll
        for (int kk = 0; kk < kVgBK; kk += 4) {
            double af[4], bf[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                af[i] = S.A[st][kk + tig][wr + i * 8 + gid];
                bf[i] = S.B[st][kk + tig][wc + i * 8 + gid];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    dmma884(acc[i][j], af[i], bf[j]);
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = r0 + wr + i * 8 + gid;
        if (r >= rows) {
            continue;
        }
        const double sg = a.top ? a.sgn[roff + r] : 1.0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                double *d = S.dst[wc + j * 8 + 2 * tig + e];
                if (d != nullptr) {
                    d[r] = acc[i][j][e] * sg;
                }
            }
        }
    }
}

// Largest K over one level's merges, for the host to size the products.
__global__ void __launch_bounds__(256) k_vec_kmax(const int *nK, int nodes, int *kmax) {
    int mx = 0;
    for (int g = threadIdx.x; g < nodes; g += blockDim.x) {
        mx = max(mx, nK[g]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(kmax, mx);
    }
}

// The top node's eigenvectors into Z (ld ldz) with the signs of E: the
// solve works on |E|, and T = S |T| S with S = diag(s), s_0 = 1,
// s_{i+1} = s_i sign(E_i) (+1 for E_i = 0), i.e. s_i = (-1)^(negative E_j,
// j < i).  One block: each thread counts the negatives of a contiguous
// chunk, a block scan gives every chunk its parity.
__global__ void __launch_bounds__(1024) k_vec_signs(const double *E, long long n, double *sgn) {
    __shared__ int iscan[32];
    const long long chunk = (n + 1023) / 1024;
    const long long lo = (long long)threadIdx.x * chunk;
    const long long hi = lo + chunk < n ? lo + chunk : n;
    int neg = 0;
    for (long long i = lo; i < hi; ++i) {
        neg += (i > 0 && E[i - 1] < 0.0) ? 1 : 0;
    }
    int tot;
    int par = block_exscan<1024>(neg, iscan, &tot);
    for (long long i = lo; i < hi; ++i) {
        par += (i > 0 && E[i - 1] < 0.0) ? 1 : 0;
        sgn[i] = (par & 1) ? -1.0 : 1.0;
    }
}

__global__ void __launch_bounds__(256) k_vec_out(const double *Q, long long ldq, long long n,
                                                 const double *sgn, double *Z, long long ldz) {
    const long long total = n * n;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long col = t / n, row = t % n;
        Z[col * ldz + row] = sgn[row] * Q[col * ldq + row];
    }
}

} // namespace brdc
