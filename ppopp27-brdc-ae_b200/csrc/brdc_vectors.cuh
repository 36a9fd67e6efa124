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
// eigenvalue index).  The two products per node are library FP64 GEMMs.
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
                    const double vx = col[rx];
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
        if (s < K + ndz) {
            add_child(vec_row_small(w, gs, s - K), 1.0);
            continue;
        }
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

// Root eigenvectors from the products (node's block of C, columns in root
// order) to their places in the node's ascending order: one warp per root.
__global__ void __launch_bounds__(256) k_vec_scatter(VArgs a, const double *C, long long total_n) {
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
        if (s >= K) {
            continue;
        }
        const int Kz = w.nKz[g];
        const int pos = vec_pos(w, gs, po, s, K, m - Kz, Kz - K);
        const double *src = C + gs * a.mstride + (long long)s * m;
        double *dst = a.top ? a.out + (long long)pos * a.ldout
                            : a.out + gs * a.out_stride + (long long)pos * m;
        for (int r = lane; r < m; r += 32) {
            dst[r] = a.top ? src[r] * a.sgn[r] : src[r];
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

// GEMM pointer tables of one level, written on the device so the level's
// products need nothing from the host: nodes have at most two sizes per
// level (the tree splits floor/ceil), so the shapes fall in up to four
// groups -- (top half, bottom half) x (smaller, larger node) -- each stored
// as A[cnt], B[cnt], C[cnt] from tab + off[group], a node's slot being its
// rank among the level's nodes of its size.  B (the node's root columns of
// M) and C (their products) sit at gstart * stride, ld m.
struct VecTables {
    long long n;
    int depth, nodes;
    int msmall, cs, cl; // smaller node size, nodes of each size
    long long off[4];
    const double *child; // the leaves' eigenvectors (ld 16) or the level below's blocks
    int leafchild;
    long long child_stride; // mmax of the level below
    const double *M;
    double *C;
    long long stride;
    const double **tab;
};

__global__ void __launch_bounds__(1024) k_vec_tables(VecTables t) {
    __shared__ int iscan[32];
    int carry = 0;
    for (int base = 0; base < t.nodes; base += 1024) {
        const int g = base + threadIdx.x;
        long long st = 0, m = 0;
        if (g < t.nodes) {
            walk_node(t.n, t.depth, g, &st, &m);
        }
        const int small = (g < t.nodes && (int)m == t.msmall) ? 1 : 0;
        int tot;
        const int ex = block_exscan<1024>(small, iscan, &tot);
        if (g < t.nodes) {
            const int rs = carry + ex;
            const int idx = small ? rs : g - rs;
            const int cnt = small ? t.cs : t.cl;
            const long long h1 = m >> 1;
            for (int half = 0; half < 2; ++half) {
                const long long cst = st + (half ? h1 : 0);
                const double *A = t.leafchild ? t.child + cst * 16 : t.child + cst * t.child_stride;
                const double *B = t.M + st * t.stride + (half ? h1 : 0);
                double *C = t.C + st * t.stride + (half ? h1 : 0);
                const long long o = t.off[(small ? 0 : 2) + half];
                t.tab[o + idx] = A;
                t.tab[o + cnt + idx] = B;
                t.tab[o + 2 * cnt + idx] = C;
            }
        }
        carry += tot;
        __syncthreads();
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
