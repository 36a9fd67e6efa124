// brdc_common.cuh -- data layout, merge-tree geometry and device helpers
// shared by the kernels and the host driver.
//
// Merge tree.  A tridiagonal of order n is cut into 2^L leaves with
// L = bitlen(n-1) - 4 for n > 16 (leaves of 8..16 rows), every node of size
// s splitting into a left child of floor(s/2) and a right child of
// ceil(s/2) rows: the tree of the reference prototype
// (gpu/src/tridiag_solver_dc.cuh:213-225, tridiag_solver_extract.cuh:63-70).
// Node starts are recomputed from the node index by walking down from the
// root (O(depth) integer steps), so no tree table lives in memory.
//
// Forest.  The batched entry solves B independent tridiagonals packed back
// to back; level k of the forest holds, for every instance b with L_b > k,
// the 2^(L_b-1-k) merges at depth L_b-1-k of that instance.  A single
// solve is a forest of one.
//
// Layout of one level's data in HBM (all arrays indexed by the global row
// index of the forest, so every node owns the contiguous slice
// [gstart, gstart+m) of each array; the pole arrays are padded so that each
// node's slice starts 16-byte aligned for cp.async.bulk):
//   cur_{d,f,l} / nxt_{d,f,l}  node eigenvalues (ascending) with the first
//                              and last rows of the node eigenvector matrix
//   m{d,z,f,l}, morig         merged child lists (sorted) with z and rows
//   a{d,z,f,l}                poles that survived the small-z test
//   z{d,f,l}, g{d,f,l}        deflated by the small-z test / by rotation
//   p{d,z,f,l}, pw            the K secular poles, their z and Loewner z
//   r{org,do,tau,lam}         per root: origin pole, d at origin, shift,
//                              eigenvalue
#pragma once

#include <cstddef>
#include <cstdint>

#include "../../include/brdc.h"

namespace brdc {

constexpr int kLeafMax = 16;
constexpr int kSweepThreads = 256;  // threads per CTA of the sweep kernels
// poles per shared-memory tile of the sweep kernel's CTA role: the largest
// multiple of 512 whose four double-buffered arrays (96 KB) still let two
// blocks share an SM; against 1024, Toeplitz 65,536 20.78 -> 20.68 ms and
// 32,768 6.46 -> 6.31 ms, the same bits (a lane's poles keep their order)
constexpr int kTile = 1536;
constexpr int kWarpMaxK = 2048;     // merges up to this K run one warp per item
constexpr double kDeflTolScale = 8.0;  // tol = 8*eps*max(max|d|,max|z|)
                                        // (merge_kernels.cuh:9-11,1090-1091)
constexpr unsigned kWsMagic = 0x42524443u; // "BRDC"
// z of a merge is the children's boundary row divided by sqrt(2), as a
// correctly rounded quotient by the correctly rounded sqrt(2), which is how
// the reference forms it (gpu/src/tridiag_solver_merge_kernels.cuh:
// 1075-1077): the same rows give the same z bit for bit, so the deflation
// decisions can be compared with the reference's exactly.
constexpr double kSqrt2 = 1.4142135623730951;

inline int tree_levels(long long n) {
    if (n <= 16) {
        return 0;
    }
    int bits = 0;
    long long r = n - 1;
    while (r > 0) {
        ++bits;
        r >>= 1;
    }
    return bits - 4;
}

// Per-level control block written by the kernels.
// Programmatic dependent launch.  Some of the solve's kernels are launched
// with the programmatic-serialization attribute, so their launch and block
// scheduling overlap the end of the kernel before them.  Every forward
// kernel starts with pdl_begin(): it lets the next kernel in the stream be
// scheduled as soon as all of this grid's CTAs are running (their resources
// are then already held, so the early CTAs only take what is left), and
// waits until the previous kernel has finished and its writes are visible.
// For a kernel launched without the attribute the wait returns at once.
__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

struct LevelCtl {
    int ticket;      // CTAs of the merge kernel that finished
    int nodes;       // merges at this level
    int tpr_w;       // lanes per root, warp-role merges (K <= kWarpMaxK)
    int tpr_c;       // lanes per root, CTA-role merges (K > kWarpMaxK)
    int items_w;     // warp work items of the level
    int items_c;     // CTA work items of the level
    int total_k;
    int nbig;        // merges k_level left to the sweep kernels (K > kLvlMaxK)
    unsigned bar_count; // grid barrier of k_sweeps: arrivals, generation
    unsigned bar_gen;
    int citem;       // next CTA-role item of the secular phase (taken by atomicAdd)
    int pad_ctl;
    double work_w;   // pole-root pairs (sum K^2) of the warp-role merges
    double work_c;   // and of the CTA-role merges
};

struct WsHeader {
    unsigned magic;
    int B;
    long long total_n;
    int max_levels;
    int flags;
    int status;      // device error code, 0 = ok
    int nonconv;     // roots that hit the iteration cap
    int leaf_sweeps_max;
    int leaf_count;
    int max_iter;    // iteration cap of one secular root (the handle's limit)
    int leaf_sweeps_sum; // Jacobi sweeps summed over the leaves
    unsigned long long wait_ns; // bound of every device-side wait, in ns
    LevelCtl lvl[BRDC_MAX_LEVELS];
    brdc_level_diagnostics diag[BRDC_MAX_LEVELS];
};

// Device error codes written to WsHeader::status.
enum DeviceError : int {
    kErrNone = 0,
    kErrBarrierTimeout = 1,     // a tile copy's mbarrier wait ran out
    kErrBadGeometry = 2,
    kErrGridBarrierTimeout = 3, // a grid-wide barrier wait ran out
    kErrNonFinite = 4,          // D or E holds a NaN or an infinity
};

// A solve whose status word is set (non-finite input, a wait that ran out)
// does no further work: every kernel after the one that set it returns at
// once.  Only k_norm and k_sweeps set the word, and every later kernel
// waits for them to finish before it reads it, so all CTAs of a kernel read
// the same value (no cluster or grid barrier can lose a member to it).
#if defined(__CUDACC__)
__device__ __forceinline__ bool halted(const WsHeader *h) {
    return *(const volatile int *)&h->status != 0;
}
#endif

// Forest description passed by value to every kernel.
struct Forest {
    int B;
    int max_levels;
    long long n0;               // B == 1: order
    int L0;                     // B == 1: levels
    const long long *off;       // [B+1] row offsets (B > 1)
    const int *lev;             // [B] levels per instance (B > 1)
    const int *node_prefix;     // [max_levels][B+1] node-count prefix (B > 1)
    const int *leaf_prefix;     // [B+1] leaf-count prefix (B > 1)
    const int *sub_prefix;      // [B+1] subtree-count prefix (B > 1)
};

// Every device array of one workspace.
struct Ws {
    WsHeader *hdr;
    // node data, ping-pong
    double *cd, *cf, *cl;
    double *nd, *nf, *nl;
    // merged lists
    double *md, *mz, *mf, *ml;
    int *morig;                  // merged position -> row within the node
    // small-z survivors, deflated lists
    double *ad, *az, *af, *al;
    int *amap;                   // active position -> merged position
    int *gmark, *gbase;          // rotated-out flag, cluster base
    int *gpos;                   // rotated-out list index -> active index
    double *gc, *gs, *gr;        // rotation of each rotated-out pole
    double *zd, *zf, *zl;
    int *zmap;                   // small-z list index -> merged position
    double *gd, *gf, *gl;
    // poles and roots (padded layout)
    double *pd, *pz, *pf, *pl, *pw;
    int *pmap;                   // pole -> active position
    int *rorg;
    double *rdo, *rtau, *rlam;
    double *rf, *rl;             // new boundary rows of each root (padded)
    // per node at one level
    int *nK, *nKz;
    double *nrho, *ntol, *nzn;
    int *pref_w, *pref_c;        // first work item of each merge (per role)
    int *items_w, *items_c;      // work item -> merge node (per role)
    // forest tables (batched)
    long long *f_off;
    int *f_lev, *f_node_prefix, *f_leaf_prefix, *f_sub_prefix;
    long long *f_norm;           // per instance: bits of max(|D|, |E|) (>= 0)
    // adjoint (present when the workspace keeps checkpoints)
    double *bcd, *bcf, *bcl, *bnd, *bnf, *bnl;   // cotangents, ping-pong
    double *bmd, *bmz, *bmf, *bml;               // at merged positions
    double *bad, *baz, *baf, *bal;               // at active positions
    double *bzd, *bzf, *bzl, *bgd, *bgf, *bgl;   // deflated lists
    double *blam, *bfr, *blr;                    // per root (padded)
    double *rinvn, *rh, *rkap, *rcdo, *rczo;     // per root (padded)
    double *rfp, *rlp;                           // per root: new rows
    double *bzz, *bgw;                           // deflated: dL/dz, dL/domega
    double *bpd, *bpz, *bpf, *bpl;               // per pole (padded)
    double *rkr;                                 // per root: its drho term
    double *wtmp;                                // eigenvalues of the re-run
    double *leafv, *leafl;                       // checkpointed leaves: eigenvectors
                                                 // (16 per row), eigenvalues
};

struct Layout {
    size_t bytes;
    long long nt;     // total rows
    long long np;     // padded pole-array length
    long long nn0;    // nodes of the widest level
    int levels;
    bool ckpt;
};

#if defined(__CUDACC__)

__host__ __device__ inline void walk_node(long long n, int depth, long long idx,
                                          long long *start, long long *size) {
    long long s = n, st = 0;
    for (int bit = depth - 1; bit >= 0; --bit) {
        const long long h = s >> 1;
        if ((idx >> bit) & 1) {
            st += h;
            s -= h;
        } else {
            s = h;
        }
    }
    *start = st;
    *size = s;
}

struct NodeGeom {
    int inst;
    int depth;        // depth of the merged node (0 = instance root)
    long long gstart; // first row of the node in the forest
    long long istart; // first row of the instance
    long long iend;   // one past the last row of the instance
    int m, m1;        // node rows, rows of the left child
    long long poff;   // aligned start of the node's pole slice
};

__device__ inline int upper_bound_int(const int *a, int n, int x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] <= x) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo;
}

__device__ inline int lower_bound_int(const int *a, int n, int x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < x) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// Geometry of merge node g (global index at forest level k).
__device__ inline NodeGeom node_geom(const Forest &F, int k, int g) {
    NodeGeom G;
    int b = 0;
    long long idx = g;
    long long n = F.n0;
    int L = F.L0;
    long long base = 0;
    if (F.B > 1) {
        const int *pre = F.node_prefix + (size_t)k * (F.B + 1);
        b = upper_bound_int(pre, F.B + 1, g) - 1;
        idx = g - pre[b];
        L = F.lev[b];
        base = F.off[b];
        n = F.off[b + 1] - base;
    }
    G.inst = b;
    G.depth = L - 1 - k;
    long long st, s;
    walk_node(n, G.depth, idx, &st, &s);
    G.gstart = base + st;
    G.istart = base;
    G.iend = base + n;
    G.m = (int)s;
    G.m1 = (int)(s >> 1);
    G.poff = (G.gstart + g + 1) & ~1LL;
    return G;
}

// Merge node at forest level k that contains global row x.  Returns false
// when the row's instance has no merge at this level.
__device__ inline bool elem_node(const Forest &F, int k, long long x, int *g,
                                 long long *gstart, int *m, int *depth_out,
                                 int *inst_out = nullptr) {
    long long base = 0, n = F.n0;
    int L = F.L0, pre = 0, inst = 0;
    if (F.B > 1) {
        int lo = 0, hi = F.B; // last b with off[b] <= x
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (F.off[mid] <= x) {
                lo = mid;
            } else {
                hi = mid;
            }
        }
        base = F.off[lo];
        n = F.off[lo + 1] - base;
        L = F.lev[lo];
        pre = F.node_prefix[(size_t)k * (F.B + 1) + lo];
        inst = lo;
    }
    if (inst_out != nullptr) {
        *inst_out = inst;
    }
    if (L <= k) {
        return false;
    }
    const int depth = L - 1 - k;
    long long st = 0, s = n, idx = 0;
    const long long r = x - base;
    for (int t = 0; t < depth; ++t) {
        const long long h = s >> 1;
        if (r - st >= h) {
            st += h;
            s -= h;
            idx = 2 * idx + 1;
        } else {
            s = h;
            idx = 2 * idx;
        }
    }
    *g = pre + (int)idx;
    *gstart = base + st;
    *m = (int)s;
    *depth_out = depth;
    return true;
}

struct LeafGeom {
    long long gstart, istart, iend;
    int s;
    int top;  // instance is a single leaf
    int inst; // instance index
};

__device__ inline LeafGeom leaf_geom(const Forest &F, long long g) {
    LeafGeom G;
    int b = 0;
    long long idx = g;
    long long n = F.n0;
    int L = F.L0;
    long long base = 0;
    if (F.B > 1) {
        b = upper_bound_int(F.leaf_prefix, F.B + 1, (int)g) - 1;
        idx = g - F.leaf_prefix[b];
        L = F.lev[b];
        base = F.off[b];
        n = F.off[b + 1] - base;
    }
    long long st, s;
    walk_node(n, L, idx, &st, &s);
    G.gstart = base + st;
    G.istart = base;
    G.iend = base + n;
    G.s = (int)s;
    G.top = (L == 0);
    G.inst = b;
    return G;
}

// Scale of instance b: matrices whose max-norm lies outside [2^-8, 2^8] are
// solved as the exact power-of-two multiple with max-norm in [0.5, 1), like
// the reference CPU path normalises before DLAED0_BR (dstedc_dc_br.f:114-128).
// The deflation tolerance mixes the scale of d with that of z (eigenvector
// entries, scale-free), so an unscaled tiny matrix would deflate every pole;
// a power of two leaves every rounding unchanged.  Returns s with D_s = s D.
__device__ inline double inst_scale(const Ws &w, int b) {
    const double mx = __longlong_as_double(w.f_norm[b]);
    if (!(mx > 0.0) || !isfinite(mx) || (mx >= 0x1.0p-8 && mx <= 0x1.0p8)) {
        return 1.0;
    }
    return ldexp(1.0, -(ilogb(mx) + 1));
}

__device__ inline double inst_unscale(const Ws &w, int b) {
    const double mx = __longlong_as_double(w.f_norm[b]);
    if (!(mx > 0.0) || !isfinite(mx) || (mx >= 0x1.0p-8 && mx <= 0x1.0p8)) {
        return 1.0;
    }
    return ldexp(1.0, ilogb(mx) + 1);
}

// ---------------------------------------------------------------- helpers

__device__ inline double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}

__device__ inline double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}

// Block-wide reductions; scratch holds >= 32 doubles.  All threads return
// the result.
template <int T>
__device__ inline double block_sum(double v, double *scratch) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        scratch[w] = v;
    }
    __syncthreads();
    double r = 0.0;
    if constexpr (T > 32) {
        r = (l < (T >> 5)) ? scratch[l] : 0.0;
        r = warp_sum(r);
    } else {
        r = scratch[0];
    }
    return r;
}

template <int T>
__device__ inline double block_max(double v, double *scratch) {
    v = warp_max(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        scratch[w] = v;
    }
    __syncthreads();
    double r;
    if constexpr (T > 32) {
        r = (l < (T >> 5)) ? scratch[l] : 0.0;
        r = warp_max(r);
    } else {
        r = scratch[0];
    }
    return r;
}

// Exclusive scan of one int per thread; *total receives the block sum.
template <int T>
__device__ inline int block_exscan(int v, int *scratch, int *total) {
    const int l = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (l >= o) {
            x += y;
        }
    }
    __syncthreads();
    if (l == 31) {
        scratch[w] = x;
    }
    __syncthreads();
    int wpre = 0, tot = 0;
    if constexpr (T > 32) {
        int s = (l < (T >> 5)) ? scratch[l] : 0;
        int inc = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc, o);
            if (l >= o) {
                inc += y;
            }
        }
        tot = __shfl_sync(0xffffffffu, inc, 31);
        wpre = __shfl_sync(0xffffffffu, inc - s, w);
    } else {
        tot = scratch[0];
    }
    *total = tot;
    return wpre + x - v;
}

// Plane rotation zeroing g against f: c*f + s*g = r >= 0, -s*f + c*g = 0
// (same convention as the reference's device_lartg,
// gpu/src/tridiag_solver_device.cuh:15-36).
__device__ inline void lartg(double f, double g, double *c, double *s,
                             double *r) {
    if (g == 0.0) {
        *c = 1.0;
        *s = 0.0;
        *r = f;
        return;
    }
    if (f == 0.0) {
        *c = 0.0;
        *s = 1.0;
        *r = g;
        return;
    }
    const double scale = fabs(f) + fabs(g);
    const double fs = f / scale, gs = g / scale;
    const double nrm = scale * sqrt(fs * fs + gs * gs);
    *c = f / nrm;
    *s = g / nrm;
    *r = nrm;
}

template <typename T>
__device__ inline int lower_bound_d(const T *a, int n, T x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < x) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo;
}

template <typename T>
__device__ inline int upper_bound_d(const T *a, int n, T x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] <= x) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// -------------------------------------------- TMA bulk copies + mbarriers
// One-dimensional cp.async.bulk global -> shared with transaction-count
// completion on an mbarrier.  Every wait is bounded in time (the handle's
// wait limit, from the workspace header): on timeout the kernel records
// kErrBarrierTimeout, waits (bounded again) for the copies it still has in
// flight, and the caller abandons the work item.

// Default bound of every device-side wait (tile copies, grid barriers):
// far above any legitimate wait (the longest grid-barrier wait of a level,
// the slowest block's share of its secular phase, is milliseconds).
constexpr unsigned long long kDefaultWaitNs = 20ull * 1000ull * 1000ull * 1000ull;
// Bound of the wait for copies still in flight after a timeout.
constexpr unsigned long long kDrainWaitNs = 2ull * 1000ull * 1000ull * 1000ull;

__device__ inline unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ inline unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ inline void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(count)
                 : "memory");
}

__device__ inline void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ inline void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Orders this thread's view of global memory written through ordinary
// stores (by this CTA or, after a cluster barrier, by its peers) before
// bulk copies it issues next, which read through the async proxy.
__device__ inline void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ inline void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile(
        "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
            smem_u32(bar)),
        "r"(bytes)
        : "memory");
}

__device__ inline void bulk_g2s(void *dst, const void *src, unsigned bytes,
                                uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Returns true when the phase completed, false when it had not after
// limit_ns (measured on %globaltimer).
__device__ inline bool mbar_wait(uint64_t *bar, unsigned phase, unsigned long long limit_ns) {
    const unsigned a = smem_u32(bar);
    const unsigned long long t0 = globaltimer_ns();
    for (;;) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(phase)
            : "memory");
        if (done) {
            return true;
        }
        if (globaltimer_ns() - t0 > limit_ns) {
            return false;
        }
    }
}

#endif // __CUDACC__

} // namespace brdc
