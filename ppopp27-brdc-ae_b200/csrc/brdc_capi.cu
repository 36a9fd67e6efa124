// brdc_capi.cu -- host driver and C ABI (include/brdc.h).
//
// The driver plans a forest (one or many tridiagonals), carves the caller's
// workspace, and enqueues the leaves and lowest levels (k_subtree), then per
// level either the fused k_level (with k_sweeps for merges that keep many
// poles) or k_merge, the deflation and k_sweeps.  All launch shapes depend
// only on the orders, never on data, and no call synchronises the stream,
// so a solve can be captured in a CUDA graph.  Data-dependent sizes (deflation counts K) travel from kernel to
// kernel through the workspace header; that replaces the per-level device
// to host copy of the reference (gpu/src/tridiag_solver.cu:624-630).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/brdc_lapack.h"
#include "brdc_backward.cuh"
#include "brdc_level.cuh"
#include "brdc_vectors.cuh"
#include "brdc_subtree.cuh"

using namespace brdc;

// A solve captured as a CUDA graph.  The graph holds every pointer and
// launch shape of one call, so it is replayed only for calls with the same
// signature.
struct SolveSig {
    int kind = 0; // 0: forward (plain or checkpointing), 1: adjoint
    long long n = 0;
    const double *D = nullptr, *E = nullptr;
    double *W = nullptr;
    void *ws = nullptr;
    size_t ws_size = 0;
    const double *srcD = nullptr, *srcE = nullptr; // host entry: mapped D, E
    const double *G = nullptr; // adjoint: G, gD, gE and keep_forward
    double *gD = nullptr, *gE = nullptr;
    int keep_forward = 0;
    int sub_levels = 0, defl_cluster = 0, lanes_target = 0, lvl_rows = 0, max_iter = 0;
    unsigned long long wait_ns = 0;
    bool operator==(const SolveSig &o) const {
        return kind == o.kind && n == o.n && D == o.D && E == o.E && W == o.W && ws == o.ws &&
               ws_size == o.ws_size && srcD == o.srcD && srcE == o.srcE && G == o.G &&
               gD == o.gD && gE == o.gE &&
               keep_forward == o.keep_forward && sub_levels == o.sub_levels &&
               defl_cluster == o.defl_cluster && lanes_target == o.lanes_target &&
               lvl_rows == o.lvl_rows && max_iter == o.max_iter && wait_ns == o.wait_ns;
    }
};

struct SolveGraph {
    SolveSig seen;                  // the last call's signature (of this kind)
    bool seen_valid = false;
    bool failed = false;            // capturing `seen` failed: no retry
    cudaGraph_t graph = nullptr;    // captured for `seen` on its second call
    cudaGraphExec_t exec = nullptr;
    // what the enqueue leaves on the host, restored by a replay
    int launches = 0;
    int fused_levels = 0;
    int timed_levels = 0;
    int has_lowner[BRDC_MAX_LEVELS] = {};
};

struct brdc_handle_struct {
    cudaStream_t own_stream;
    cudaStream_t stream;
    int last_code;
    brdc_error_source last_src;
    const char *last_site;
    int sm_count;
    int device;
    // batched: signature of the forest whose tables the last non-captured
    // batched call wrote into a workspace, the host copy of those tables
    // (alive until their copy has run, prep_ev) and the event itself
    const void *prep_ws;
    bool prep_ckpt = false;
    int prep_sub = -1;
    std::vector<int> prep_tab;
    cudaEvent_t prep_ev = nullptr;
    bool prep_pending = false;
    // merge levels solved inside the subtree kernel (0: leaves alone,
    // -1: chosen per solve from the tree height)
    int sub_levels = -1;
    int defl_cluster = 16;        // largest deflation cluster (8 for k_merge_deflate_cl)
    int lanes_target = 303104;    // root-sweep parallelism target
    int lvl_rows = 1 << 30;       // largest merge of a level run by k_level (0: none)
    // failure limits (brdc_set_limits): secular iteration cap, device wait bound
    int max_iter = kSecularMaxIter;
    unsigned long long wait_ns = kDefaultWaitNs;
    std::vector<long long> prep_off;
    // phase timing (off by default)
    int timing;
    cudaEvent_t ev[2 + 4 * BRDC_MAX_LEVELS + 2];
    int ev_ready;
    int ev_used;
    int launches;
    int timed_levels;
    int has_lowner[BRDC_MAX_LEVELS];
    int fused_levels;
    // graph replay of repeated solves (brdc_set_graphs): one graph for the
    // forwards, one for the adjoints, so that a forward-and-adjoint loop
    // replays both; the stream they are captured on (the caller's may be
    // the legacy stream, which cannot be captured)
    int graphs = 1;
    SolveGraph gf, gb;
    cudaStream_t gcap = nullptr;
    bool replayed = false;          // the last solve was a replay
};

namespace {

void set_error(brdc_handle h, int code, brdc_error_source src,
               const char *site) {
    if (h != nullptr) {
        h->last_code = code;
        h->last_src = src;
        h->last_site = site;
    }
}

#define BRDC_CUDA(h, site, expr)                                               \
    do {                                                                       \
        const cudaError_t e__ = (expr);                                        \
        if (e__ != cudaSuccess) {                                              \
            set_error((h), (int)e__, BRDC_ERROR_SRC_CUDA, (site));             \
            return BRDC_STATUS_CUDA_ERROR;                                     \
        }                                                                      \
    } while (0)

constexpr size_t kAlign = 256; // gpu/src/workspace_align.hpp:9
// largest order of the eigenvector path (n^2 doubles of eigenvectors, 2 n^2 of work)
constexpr long long kMaxVectorOrder = 32768;

size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// Subtrees of an instance with L merge levels when the subtree kernel
// takes its lowest `fused` levels.
long long subtrees_of(int L, int fused) {
    const int Ls = L < fused ? L : fused;
    return 1LL << (L - Ls);
}

// Host view of a forest.
struct HostForest {
    int B = 0;
    std::vector<long long> off;  // B+1
    std::vector<int> lev;        // B
    int max_levels = 0;
    long long total_n = 0;
    long long leaves = 0;
    std::vector<int> level_nodes; // nodes per level
    std::vector<int> level_mmax;  // largest node per level
    std::vector<long long> level_rows; // rows of instances merging at a level
    long long nn0 = 0;            // max nodes of a level
};

bool build_forest(int B, const long long *off, HostForest *f) {
    f->B = B;
    f->off.assign(off, off + B + 1);
    f->lev.resize(B);
    f->max_levels = 0;
    f->leaves = 0;
    f->total_n = off[B] - off[0];
    for (int b = 0; b < B; ++b) {
        const long long n = off[b + 1] - off[b];
        if (n <= 0 || n > (1LL << 30)) {
            return false;
        }
        f->lev[b] = tree_levels(n);
        f->max_levels = std::max(f->max_levels, f->lev[b]);
        f->leaves += 1LL << f->lev[b];
    }
    if (f->max_levels >= BRDC_MAX_LEVELS) {
        return false;
    }
    f->level_nodes.assign(f->max_levels, 0);
    f->level_mmax.assign(f->max_levels, 0);
    f->level_rows.assign(f->max_levels, 0);
    for (int b = 0; b < B; ++b) {
        const long long n = off[b + 1] - off[b];
        const int L = f->lev[b];
        for (int k = 0; k < L; ++k) {
            const int depth = L - 1 - k;
            f->level_nodes[k] += 1 << depth;
            f->level_rows[k] += n;
            const long long mm = (n + (1LL << depth) - 1) >> depth;
            f->level_mmax[k] = std::max<long long>(f->level_mmax[k], mm);
        }
    }
    f->nn0 = 1;
    for (int k = 0; k < f->max_levels; ++k) {
        f->nn0 = std::max<long long>(f->nn0, f->level_nodes[k]);
    }
    return true;
}

// Workspace descriptor: every array with its element size, its length
// class and whether a checkpointing workspace keeps one slice per level
// (the arrays the adjoint reads back).
enum CountKind { CN_NT, CN_NT16, CN_NP, CN_NN, CN_NN1, CN_ITW, CN_ITC, CN_B1, CN_B, CN_NODEPRE,
                 CN_INST };

struct SlotDesc {
    int kind;        // 0 double*, 1 int*, 2 long long*
    double *Ws::*fd;
    int *Ws::*fi;
    long long *Ws::*fl;
    CountKind count;
    bool per_level;
    bool adjoint;
};

#define SD(field, cnt, pl, adj) {0, &Ws::field, nullptr, nullptr, cnt, pl, adj}
#define SI(field, cnt, pl, adj) {1, nullptr, &Ws::field, nullptr, cnt, pl, adj}
#define SL(field, cnt, pl, adj) {2, nullptr, nullptr, &Ws::field, cnt, pl, adj}

const SlotDesc kSlots[] = {
    SD(cd, CN_NT, false, false), SD(cf, CN_NT, false, false), SD(cl, CN_NT, false, false),
    SD(nd, CN_NT, false, false), SD(nf, CN_NT, false, false), SD(nl, CN_NT, false, false),
    SD(md, CN_NT, true, false), SD(mz, CN_NT, true, false), SD(mf, CN_NT, false, false),
    SD(ml, CN_NT, false, false), SI(morig, CN_NT, true, false),
    SD(ad, CN_NT, false, false), SD(az, CN_NT, false, false), SD(af, CN_NT, true, false),
    SD(al, CN_NT, true, false), SI(amap, CN_NT, true, false), SI(gmark, CN_NT, true, false),
    SI(gbase, CN_NT, true, false), SI(gpos, CN_NT, true, false), SD(gc, CN_NT, true, false), SD(gs, CN_NT, true, false),
    SD(gr, CN_NT, true, false),
    SD(zd, CN_NT, true, false), SD(zf, CN_NT, true, false), SD(zl, CN_NT, true, false),
    SI(zmap, CN_NT, true, false),
    SD(gd, CN_NT, true, false), SD(gf, CN_NT, false, false), SD(gl, CN_NT, false, false),
    SD(pd, CN_NP, true, false), SD(pz, CN_NP, true, false), SD(pf, CN_NP, true, false),
    SD(pl, CN_NP, true, false), SD(pw, CN_NP, true, false), SI(pmap, CN_NP, true, false),
    SI(rorg, CN_NP, true, false), SD(rdo, CN_NP, true, false), SD(rtau, CN_NP, true, false),
    SD(rlam, CN_NP, true, false), SD(rf, CN_NP, false, false), SD(rl, CN_NP, false, false),
    SI(nK, CN_NN, true, false), SI(nKz, CN_NN, true, false), SD(nrho, CN_NN, true, false),
    SD(ntol, CN_NN, true, false), SD(nzn, CN_NN, false, false),
    SI(pref_w, CN_NN1, true, false), SI(pref_c, CN_NN1, true, false),
    SI(items_w, CN_ITW, true, false), SI(items_c, CN_ITC, true, false),
    SL(f_off, CN_B1, false, false), SI(f_lev, CN_B, false, false),
    SI(f_node_prefix, CN_NODEPRE, false, false), SI(f_leaf_prefix, CN_B1, false, false),
    SI(f_sub_prefix, CN_B1, false, false), SL(f_norm, CN_INST, false, false),
    // adjoint
    SD(bcd, CN_NT, false, true), SD(bcf, CN_NT, false, true), SD(bcl, CN_NT, false, true),
    SD(bnd, CN_NT, false, true), SD(bnf, CN_NT, false, true), SD(bnl, CN_NT, false, true),
    SD(bmd, CN_NT, false, true), SD(bmz, CN_NT, false, true), SD(bmf, CN_NT, false, true),
    SD(bml, CN_NT, false, true), SD(bad, CN_NT, false, true), SD(baz, CN_NT, false, true),
    SD(baf, CN_NT, false, true), SD(bal, CN_NT, false, true), SD(bzd, CN_NT, false, true),
    SD(bzf, CN_NT, false, true), SD(bzl, CN_NT, false, true), SD(bgd, CN_NT, false, true),
    SD(bgf, CN_NT, false, true), SD(bgl, CN_NT, false, true),
    SD(blam, CN_NP, false, true), SD(bfr, CN_NP, false, true), SD(blr, CN_NP, false, true),
    SD(rinvn, CN_NP, false, true), SD(rh, CN_NP, false, true), SD(rkap, CN_NP, false, true),
    SD(rcdo, CN_NP, false, true), SD(rczo, CN_NP, false, true),
    SD(rfp, CN_NP, false, true), SD(rlp, CN_NP, false, true),
    SD(bzz, CN_NT, false, true), SD(bgw, CN_NT, false, true),
    SD(bpd, CN_NP, false, true), SD(bpz, CN_NP, false, true), SD(bpf, CN_NP, false, true),
    SD(bpl, CN_NP, false, true), SD(rkr, CN_NP, false, true), SD(wtmp, CN_NT, false, true),
    SD(leafv, CN_NT16, false, true), SD(leafl, CN_NT, false, true),
};

long long slot_count(CountKind c, const HostForest &f, const Layout &L) {
    switch (c) {
    case CN_NT: return L.nt;
    case CN_NT16: return 16 * L.nt;
    case CN_NP: return L.np;
    case CN_NN: return L.nn0;
    case CN_NN1: return L.nn0 + 1;
    case CN_ITW: return L.nt + L.nn0 + 2;
    case CN_ITC: return L.nt / 8 + L.nn0 + 2;
    case CN_B1: return f.B > 1 ? f.B + 1 : 0;
    case CN_B: return f.B > 1 ? f.B : 0;
    case CN_NODEPRE: return f.B > 1 ? (long long)(f.B + 1) * std::max(f.max_levels, 1) : 0;
    case CN_INST: return std::max(f.B, 1);
    }
    return 0;
}

// Compute the layout; when base is given, also point every Ws array at it.
Layout plan_workspace(const HostForest &f, bool ckpt, void *base, Ws *w) {
    Layout L{};
    L.nt = f.total_n;
    L.nn0 = f.nn0;
    // even, so that every level's slice of a checkpointing workspace keeps
    // the pole slices 16-byte aligned for the bulk copies
    L.np = (f.total_n + f.nn0 + 4 + 1) & ~1LL;
    L.levels = f.max_levels;
    L.ckpt = ckpt;
    size_t cur = align_up(sizeof(WsHeader));
    char *b = static_cast<char *>(base);
    if (w != nullptr) {
        *w = Ws{};
        w->hdr = reinterpret_cast<WsHeader *>(b);
    }
    for (const SlotDesc &sd : kSlots) {
        if (sd.adjoint && !ckpt) {
            continue;
        }
        const long long cnt = slot_count(sd.count, f, L);
        if (cnt == 0) {
            continue;
        }
        const size_t elem = sd.kind == 0 ? sizeof(double) : (sd.kind == 1 ? sizeof(int) : sizeof(long long));
        const long long reps = (ckpt && sd.per_level) ? std::max(f.max_levels, 1) : 1;
        if (w != nullptr) {
            char *p = b + cur;
            if (sd.kind == 0) {
                w->*(sd.fd) = reinterpret_cast<double *>(p);
            } else if (sd.kind == 1) {
                w->*(sd.fi) = reinterpret_cast<int *>(p);
            } else {
                w->*(sd.fl) = reinterpret_cast<long long *>(p);
            }
        }
        cur = align_up(cur + elem * (size_t)cnt * (size_t)reps);
    }
    L.bytes = align_up(cur);
    return L;
}

// Point the checkpointed arrays of *w at level k's slice.
void level_view(const HostForest &f, const Layout &L, const Ws &base, int k, Ws *w) {
    if (!L.ckpt) {
        return;
    }
    for (const SlotDesc &sd : kSlots) {
        if (!sd.per_level || sd.adjoint) {
            continue;
        }
        const long long cnt = slot_count(sd.count, f, L);
        if (sd.kind == 0) {
            w->*(sd.fd) = base.*(sd.fd) + (size_t)k * (size_t)cnt;
        } else if (sd.kind == 1) {
            w->*(sd.fi) = base.*(sd.fi) + (size_t)k * (size_t)cnt;
        }
    }
}

Layout make_layout(const HostForest &f, bool ckpt = false) {
    return plan_workspace(f, ckpt, nullptr, nullptr);
}

Ws carve(void *base, const HostForest &f, bool ckpt) {
    Ws w;
    plan_workspace(f, ckpt, base, &w);
    return w;
}

template <int T>
void launch_md(const KArgs &a, int grid, cudaStream_t s) {
    k_merge_deflate<T><<<grid, T, 0, s>>>(a);
}

// Programmatic dependent launch (the kernels begin with pdl_begin): the
// launch and block scheduling of a solve kernel overlap the end of the one
// before it in the stream.  Used for k_norm, k_level and k_plan, whose CTAs
// take whole SMs or are few (1-2.6% off the solve at n = 4096-65,536).
cudaLaunchAttribute pdl_attr() {
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at.val.programmaticStreamSerializationAllowed = 1;
    return at;
}

cudaLaunchConfig_t plain_config(unsigned grid, unsigned block, size_t smem, cudaStream_t s,
                                cudaLaunchAttribute *at) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    at[0] = pdl_attr();
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cfg;
}

cudaLaunchConfig_t cluster_config(unsigned grid, int C, cudaStream_t s, cudaLaunchAttribute *at) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(1024);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cfg;
}

// Largest cluster (8, 4, 2) of 1024-thread deflation CTAs the device can
// schedule; 1 when none.  Asked once per device.
int max_defl_cluster(int device) {
    static int cached[64];
    static bool done[64];
    if (device < 0 || device >= 64) {
        return 1;
    }
    if (!done[device]) {
        int best = 1;
        for (int C = 8; C >= 2; C >>= 1) {
            cudaLaunchAttribute at[1];
            cudaLaunchConfig_t cfg = cluster_config((unsigned)C, C, nullptr, at);
            int n = 0;
            if (cudaOccupancyMaxActiveClusters(&n, k_merge_deflate_cl<1024>, &cfg) == cudaSuccess &&
                n > 0) {
                best = C;
                break;
            }
            cudaGetLastError();
        }
        cached[device] = best;
        done[device] = true;
    }
    return cached[device];
}

// Returns the number of kernels launched.
int launch_merge_deflate(brdc_handle h, const KArgs &a0, int mmax, cudaStream_t s) {
    // about 4 rows per thread, 32..1024 threads
    int t = 32;
    while (t < 1024 && t * 4 < mmax) {
        t <<= 1;
    }
    // merges of two or more 4096-row chunks: a cluster of CTAs per node
    const int chunk = kDeflEPT * 1024;
    if (mmax >= 2 * chunk) {
        const int C = std::min(std::min(max_defl_cluster(h->device), h->defl_cluster),
                               std::min(8, mmax / chunk));
        if (C >= 2) {
            KArgs a = a0;
            a.plan_inline = a.nodes <= 1024 ? 1 : 0;
            cudaLaunchAttribute at[1];
            cudaLaunchConfig_t cfg = cluster_config((unsigned)(a.nodes * C), C, s, at);
            cudaLaunchKernelEx(&cfg, k_merge_deflate_cl<1024>, a);
            if (!a.plan_inline) {
                k_plan<1024><<<1, 1024, 0, s>>>(a);
                return 2;
            }
            return 1;
        }
    }
    // the level plan walks every node; the last deflation CTA does it while
    // that is at most one node per thread, a 1024-thread k_plan otherwise
    KArgs a = a0;
    a.plan_inline = a.nodes <= t ? 1 : 0;
    switch (t) {
    case 32: launch_md<32>(a, a.nodes, s); break;
    case 64: launch_md<64>(a, a.nodes, s); break;
    case 128: launch_md<128>(a, a.nodes, s); break;
    case 256: launch_md<256>(a, a.nodes, s); break;
    case 512: launch_md<512>(a, a.nodes, s); break;
    default: launch_md<1024>(a, a.nodes, s); break;
    }
    if (!a.plan_inline) {
        k_plan<1024><<<1, 1024, 0, s>>>(a);
        return 2;
    }
    return 1;
}

constexpr size_t smem_tiles(int na) { return sizeof(double) * 2 * na * kTile; }

bool g_attr_done = false;

cudaError_t set_attrs() {
    if (g_attr_done) {
        return cudaSuccess;
    }
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) {
        e = cudaFuncSetAttribute(k_subtree<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(SubSmem<256>));
    }
    if (e == cudaSuccess) {
        e = cudaFuncSetAttribute(k_subtree<512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(SubSmem<512>));
    }
    if (e == cudaSuccess) {
        e = cudaFuncSetAttribute(k_level<kLvlThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(LvlSmem));
    }
    if (e == cudaSuccess) {
        e = cudaFuncSetAttribute(k_level<kLvlThreads>,
                                 cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    }
    if (e == cudaSuccess) {
        e = cudaFuncSetAttribute(k_sweeps, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_tiles(4));
    }
    g_attr_done = (e == cudaSuccess);
    return e;
}

// Event slot layout of one timed solve: 0 before init, 1 after init,
// 2 after the leaves, then 4 per level (after merge, secular, lowner, rows).
void mark(brdc_handle h, int slot) {
    if (h->timing && h->ev_ready) {
        cudaEventRecord(h->ev[slot], h->stream);
        h->ev_used = std::max(h->ev_used, slot + 1);
    }
}

// Subtree depth of a solve: the handle's setting, or by default the depth
// measured fastest on B200: 5 for a batch with at least two 512-row
// subtrees per SM (the subtrees fill the GPU), otherwise by the forest's
// tallest instance (3 up to 11 levels, i.e. n <= 32768; 5 above).
int effective_sub_levels(brdc_handle h, const HostForest &hf) {
    if (h->sub_levels >= 0) {
        return h->sub_levels;
    }
    if (hf.B > 1 && hf.total_n >= 512LL * 2 * h->sm_count) {
        return 5;
    }
    // measured on B200 (uniform and normal, ms per solve): depth 3 is the
    // fastest up to n = 32,768 (11 levels; 32,768: 0.583 against 0.609 at
    // depth 4), depth 5 from 49,152 on (49,152: 0.695 against 0.718)
    return hf.max_levels <= 11 ? 3 : 5;
}

// Clusters of C = 1, 2, 4, 8, 16 k_level CTAs the device holds at once
// (0: C not schedulable).  Asked once per device (after set_attrs, which
// sizes its shared memory and allows the non-portable size 16).
const int *level_clusters(int device) {
    static int cached[64][5];
    static bool done[64];
    static const int none[5] = {0, 0, 0, 0, 0};
    if (device < 0 || device >= 64) {
        return none;
    }
    if (!done[device]) {
        for (int q = 0; q < 5; ++q) {
            const int C = 1 << q;
            cudaLaunchAttribute at[1];
            cudaLaunchConfig_t cfg = cluster_config((unsigned)C, C, nullptr, at);
            cfg.blockDim = dim3(kLvlThreads);
            cfg.dynamicSmemBytes = sizeof(LvlSmem);
            int n = 0;
            if (cudaOccupancyMaxActiveClusters(&n, k_level<kLvlThreads>, &cfg) != cudaSuccess) {
                cudaGetLastError();
                n = 0;
            }
            cached[device][q] = n;
        }
        done[device] = true;
    }
    return cached[device];
}

// Resident k_sweeps blocks per SM (without / with the CTA-role tiles), once
// per device; 0 when the device has no cooperative launch.
int sweeps_per_sm(int device, bool tiles) {
    static int cached[64][2];
    static bool done[64][2];
    if (device < 0 || device >= 64) {
        return 0;
    }
    if (!done[device][tiles]) {
        int coop = 0, nb = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
        if (coop == 0 ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_sweeps, kSweepThreads,
                                                          tiles ? smem_tiles(4) : 0) !=
                cudaSuccess) {
            cudaGetLastError();
            nb = 0;
        }
        cached[device][tiles] = nb;
        done[device][tiles] = true;
    }
    return cached[device][tiles];
}

// Roots, Loewner weights, rows and placement of level a.k: one cooperative
// k_sweeps (with tile memory where a merge can exceed kWarpMaxK poles).
// Returns the number of kernels launched, or -1 where the device cannot
// launch a cooperative grid (every sm_100 device can).
int launch_sweeps(brdc_handle h, const HostForest &hf, const KArgs &a, cudaStream_t s) {
    const int k = a.k;
    const bool tiles = hf.level_mmax[k] > kWarpMaxK;
    const int rows = h->has_lowner[k];
    const int nb = sweeps_per_sm(h->device, tiles);
    if (nb <= 0) {
        return -1;
    }
    const int grid = nb * h->sm_count;
    // an ordinary (not programmatic) cooperative launch: it measured no
    // faster with the programmatic attribute
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kSweepThreads);
    cfg.dynamicSmemBytes = tiles ? smem_tiles(4) : 0;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_sweeps, a, tiles ? 1 : 0, rows, (long long)hf.total_n);
    mark(h, 4 + 4 * k);
    mark(h, 5 + 4 * k);
    mark(h, 6 + 4 * k);
    return 1;
}

// One fused level (k_level), then k_sweeps for its merges with more than
// kLvlMaxK poles (it returns at once when there are none; it is not launched
// where no merge has more rows than that).  Returns the number of kernels
// launched.
int launch_level_fused(brdc_handle h, const HostForest &hf, const KArgs &a0, bool ckpt,
                       cudaStream_t s) {
    const int k = a0.k;
    const int mmax = hf.level_mmax[k];
    // a cluster per node: at least one CTA per kLvlRowsPerCta rows, then
    // larger while every node's cluster still runs in the first wave
    const int *act = level_clusters(h->device);
    int q = 0;
    while (q < 4 && (1 << q) < h->defl_cluster && act[q + 1] > 0 &&
           (1 << q) * kLvlRowsPerCta < mmax) {
        ++q;
    }
    while (q < 4 && (2 << q) <= h->defl_cluster && act[q + 1] >= a0.nodes) {
        ++q;
    }
    const int C = 1 << q;
    KArgs a = a0;
    a.big_k = kLvlMaxK;
    // a plan is needed only where a merge can keep more than kLvlMaxK poles
    const bool big = mmax > kLvlMaxK;
    a.plan_inline = big && a.nodes <= kLvlThreads ? 1 : 0;
    cudaLaunchAttribute at[2];
    cudaLaunchConfig_t cfg = cluster_config((unsigned)(a.nodes * C), C, s, at);
    cfg.blockDim = dim3(kLvlThreads);
    cfg.dynamicSmemBytes = sizeof(LvlSmem);
    at[1] = pdl_attr();
    cfg.numAttrs = 2;
    cudaLaunchKernelEx(&cfg, k_level<kLvlThreads>, a);
    int n = 1;
    if (big && !a.plan_inline) {
        cudaLaunchAttribute pa[1];
        cudaLaunchConfig_t pc = plain_config(1, 1024, 0, s, pa);
        cudaLaunchKernelEx(&pc, k_plan<1024>, a);
        ++n;
    }
    mark(h, 3 + 4 * k);
    if (big) {
        const int ns = launch_sweeps(h, hf, a, s);
        if (ns < 0) {
            return -1;
        }
        n += ns;
    } else {
        // no merge of this level can keep more than kLvlMaxK poles
        mark(h, 4 + 4 * k);
        mark(h, 5 + 4 * k);
        mark(h, 6 + 4 * k);
    }
    (void)ckpt; // the adjoint's full plan of this level comes with run_forest's last launch
    return n;
}

// Enqueue the whole forward solve.
brdc_status run_forest(brdc_handle h, const HostForest &hf, const Layout &L,
                       const Forest &F, const Ws &w, const double *D,
                       const double *E, double *W, const double *srcD = nullptr,
                       const double *srcE = nullptr) {
    cudaStream_t s = h->stream;
    BRDC_CUDA(h, "brdc.set_attributes", set_attrs());
    h->replayed = false;
    h->ev_used = 0;
    h->launches = 0;
    h->timed_levels = hf.max_levels;
    mark(h, 0);
    k_init<<<1, 64, 0, s>>>(w.hdr, hf.max_levels, hf.B, hf.total_n, hf.leaves, 0, w.f_norm,
                            h->max_iter, h->wait_ns);
    BRDC_CUDA(h, "brdc.init", cudaGetLastError());
    {
        long long ng = hf.B > 1 ? (hf.B + 7) / 8 : (hf.total_n + 255) / 256;
        ng = std::max<long long>(1, std::min<long long>(ng, (long long)h->sm_count * 4));
        cudaLaunchAttribute at[1];
        cudaLaunchConfig_t cfg = plain_config((unsigned)ng, 256, 0, s, at);
        cudaLaunchKernelEx(&cfg, k_norm, F, srcD ? srcD : D, srcD ? srcE : E, w.f_norm, w.hdr,
                           srcD ? const_cast<double *>(D) : (double *)nullptr,
                           srcD ? const_cast<double *>(E) : (double *)nullptr);
        BRDC_CUDA(h, "brdc.norm", cudaGetLastError());
    }
    h->launches += 2;
    mark(h, 1);

    KArgs a{};
    a.F = F;
    a.w = w;
    a.D = D;
    a.E = E;
    a.W = W;
    a.lanes_target = h->lanes_target;
    // leaves and the lowest merge levels; a checkpointing forward solves the
    // leaves first, keeping their whole eigenvector matrices for the adjoint
    const int sub = effective_sub_levels(h, hf);
    const int fused = std::min(sub, hf.max_levels);
    const long long leaf_per = 2LL * kLeafWarps; // leaves per block
    long long leaf_grid = (hf.leaves + leaf_per - 1) / leaf_per;
    leaf_grid = std::max<long long>(1, std::min<long long>(leaf_grid, (long long)h->sm_count * 16));
    if (L.ckpt) {
        k_leaf_full<<<(unsigned)leaf_grid, kLeafWarps * 32, 0, s>>>(a, hf.leaves);
        BRDC_CUDA(h, "brdc.leaf_full", cudaGetLastError());
        ++h->launches;
    }
    if (sub > 0) {
        SubArgs A{};
        A.a = a;
        for (int k = 0; k < fused; ++k) {
            A.lw[k] = w;
            level_view(hf, L, w, k, &A.lw[k]);
        }
        // the first per-level merge (level `fused`) reads the buffer that
        // `fused` ping-pong swaps leave in the child slot
        A.out_d = (fused & 1) ? w.nd : w.cd;
        A.out_f = (fused & 1) ? w.nf : w.cf;
        A.out_l = (fused & 1) ? w.nl : w.cl;
        A.levels = sub;
        A.ckpt = L.ckpt ? 1 : 0;
        A.leaves_done = L.ckpt ? 1 : 0;
        long long subs = 0;
        for (int b = 0; b < hf.B; ++b) {
            subs += subtrees_of(hf.lev[b], sub);
        }
        // an ordinary launch: scheduled while k_norm still ran (programmatic
        // launch), the subtree CTAs landed on the SMs free at that moment
        // and the subtree phase took 4-6% longer at n = 16,384-32,768
        if (sub_rows_for(sub) == 256) {
            k_subtree<256><<<(unsigned)subs, 256, sizeof(SubSmem<256>), s>>>(A);
        } else {
            k_subtree<512><<<(unsigned)subs, 512, sizeof(SubSmem<512>), s>>>(A);
        }
        BRDC_CUDA(h, "brdc.subtree", cudaGetLastError());
        ++h->launches;
        mark(h, 2);
        for (int k = 0; k < fused; ++k) {
            h->has_lowner[k] = 0;
        }
        h->fused_levels = fused;
        if (fused & 1) {
            std::swap(a.w.cd, a.w.nd);
            std::swap(a.w.cf, a.w.nf);
            std::swap(a.w.cl, a.w.nl);
        }
    } else {
        if (!L.ckpt) {
            k_leaf<<<(unsigned)leaf_grid, kLeafWarps * 32, 0, s>>>(a, hf.leaves);
            BRDC_CUDA(h, "brdc.leaf", cudaGetLastError());
            ++h->launches;
        }
        mark(h, 2);
        h->fused_levels = 0;
    }
    long long elem_grid = (hf.total_n + 255) / 256;
    elem_grid = std::max<long long>(1, std::min<long long>(elem_grid, (long long)h->sm_count * 8));
    for (int k = (sub > 0 ? fused : 0); k < hf.max_levels; ++k) {
        a.k = k;
        a.nodes = hf.level_nodes[k];
        a.level_rows = hf.level_rows[k];
        level_view(hf, L, w, k, &a.w);
        // rows are needed unless every merge of this level is an instance root
        bool any_inner = false;
        for (int b = 0; b < hf.B; ++b) {
            if (hf.lev[b] - 1 > k) {
                any_inner = true;
                break;
            }
        }
        h->has_lowner[k] = any_inner ? 1 : 0;
        int nl;
        if (hf.level_mmax[k] <= h->lvl_rows) {
            nl = launch_level_fused(h, hf, a, L.ckpt, s);
            BRDC_CUDA(h, "brdc.level", cudaGetLastError());
        } else {
            k_merge<<<(unsigned)elem_grid, 256, 0, s>>>(a, hf.total_n);
            BRDC_CUDA(h, "brdc.merge", cudaGetLastError());
            h->launches += 1 + launch_merge_deflate(h, a, hf.level_mmax[k], s);
            BRDC_CUDA(h, "brdc.merge_deflate", cudaGetLastError());
            mark(h, 3 + 4 * k);
            nl = launch_sweeps(h, hf, a, s);
            BRDC_CUDA(h, "brdc.sweeps", cudaGetLastError());
        }
        if (nl < 0) {
            set_error(h, (int)cudaErrorNotSupported, BRDC_ERROR_SRC_CUDA,
                      "brdc.sweeps: no cooperative launch on this device");
            return BRDC_STATUS_NOT_IMPLEMENTED;
        }
        h->launches += nl;
        std::swap(a.w.cd, a.w.nd);
        std::swap(a.w.cf, a.w.nf);
        std::swap(a.w.cl, a.w.nl);
    }
    if (L.ckpt) {
        // the item tables of every merge on the levels the forward solved
        // without them (subtree and fused levels), which the adjoint's
        // sweeps read: one launch, one CTA per level
        static_assert(sizeof(PlanAllArgs) <= 4096, "kernel parameters of k_plan_all");
        PlanAllArgs P{};
        P.base = a;
        int cnt = 0;
        for (int k = 0; k < hf.max_levels && cnt < kPlanMaxLevels; ++k) {
            const bool sub_level = sub > 0 && k < fused;
            const bool fused_level = !sub_level && hf.level_mmax[k] <= h->lvl_rows;
            if (!sub_level && !fused_level) {
                continue;
            }
            Ws v = w;
            level_view(hf, L, w, k, &v);
            PlanLevel &pl = P.lv[cnt++];
            pl.nK = v.nK;
            pl.nKz = v.nKz;
            pl.pref_w = v.pref_w;
            pl.pref_c = v.pref_c;
            pl.items_w = v.items_w;
            pl.items_c = v.items_c;
            pl.nodes = hf.level_nodes[k];
            pl.k = k;
            pl.rows = hf.level_rows[k];
        }
        if (cnt > 0) {
            k_plan_all<1024><<<cnt, 1024, 0, s>>>(P);
            BRDC_CUDA(h, "brdc.plans", cudaGetLastError());
            ++h->launches;
        }
    }
    return BRDC_STATUS_SUCCESS;
}

void drop_graph(SolveGraph &g) {
    if (g.exec != nullptr) {
        cudaGraphExecDestroy(g.exec);
    }
    if (g.graph != nullptr) {
        cudaGraphDestroy(g.graph);
    }
    g.exec = nullptr;
    g.graph = nullptr;
}

// Capture what enqueue() launches into g and instantiate it.  On any
// failure nothing is kept, the handle's error state is as before, and the
// caller launches the solve as usual.
template <class Enqueue>
bool capture_graph(brdc_handle h, SolveGraph &g, Enqueue enqueue) {
    const int code = h->last_code;
    const brdc_error_source src = h->last_src;
    const char *site = h->last_site;
    auto fail = [&]() {
        cudaGetLastError();
        h->last_code = code;
        h->last_src = src;
        h->last_site = site;
        return false;
    };
    if (set_attrs() != cudaSuccess) {
        return fail();
    }
    if (h->gcap == nullptr &&
        cudaStreamCreateWithFlags(&h->gcap, cudaStreamNonBlocking) != cudaSuccess) {
        h->gcap = nullptr;
        return fail();
    }
    cudaGraph_t graph = nullptr;
    if (cudaGraphCreate(&graph, 0) != cudaSuccess) {
        return fail();
    }
    if (cudaStreamBeginCaptureToGraph(h->gcap, graph, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGraphDestroy(graph);
        return fail();
    }
    // the graph records kernels only, so the stream it is captured on does
    // not matter for its replays on the caller's stream
    cudaStream_t user = h->stream;
    h->stream = h->gcap;
    const brdc_status st = enqueue();
    h->stream = user;
    cudaGraph_t out = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(h->gcap, &out);
    cudaGraphExec_t exec = nullptr;
    if (st != BRDC_STATUS_SUCCESS || ec != cudaSuccess || out != graph ||
        cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
        if (exec != nullptr) {
            cudaGraphExecDestroy(exec);
        }
        cudaGraphDestroy(graph);
        return fail();
    }
    g.graph = graph;
    g.exec = exec;
    g.launches = h->launches;
    g.fused_levels = h->fused_levels;
    g.timed_levels = h->timed_levels;
    std::copy(h->has_lowner, h->has_lowner + BRDC_MAX_LEVELS, g.has_lowner);
    return true;
}

// A solve as a graph replay, when this call repeats the previous call's
// signature of its kind (pointers, order, workspace, tuning and limits):
// captured on that second call, replayed from then on.  A replay runs the
// same kernels with the same arguments and programmatic edges, and saves
// the launch processing of each (uniform 65,536 on B200: 0.742 -> 0.725 ms).
// *done = false hands the call to the ordinary launches: replay switched
// off, phase timing on, a stream the caller is capturing (its own graph
// then holds the launches), the first call of a signature, or a failed
// capture.
template <class Enqueue>
brdc_status graph_call(brdc_handle h, SolveGraph &g, SolveSig sig, Enqueue enqueue,
                       bool *done) {
    *done = false;
    h->replayed = false;
    if (!h->graphs || h->timing) {
        return BRDC_STATUS_SUCCESS;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(h->stream, &cs) != cudaSuccess) {
        cudaGetLastError();
        return BRDC_STATUS_SUCCESS;
    }
    if (cs != cudaStreamCaptureStatusNone) {
        return BRDC_STATUS_SUCCESS;
    }
    sig.sub_levels = h->sub_levels;
    sig.defl_cluster = h->defl_cluster;
    sig.lanes_target = h->lanes_target;
    sig.lvl_rows = h->lvl_rows;
    sig.max_iter = h->max_iter;
    sig.wait_ns = h->wait_ns;
    if (!(g.seen_valid && g.seen == sig)) {
        drop_graph(g);
        g.seen = sig;
        g.seen_valid = true;
        g.failed = false;
        return BRDC_STATUS_SUCCESS;
    }
    if (g.failed) {
        return BRDC_STATUS_SUCCESS;
    }
    if (g.exec == nullptr && !capture_graph(h, g, enqueue)) {
        g.failed = true;
        return BRDC_STATUS_SUCCESS;
    }
    *done = true;
    h->ev_used = 0;
    h->launches = g.launches;
    h->fused_levels = g.fused_levels;
    h->timed_levels = g.timed_levels;
    std::copy(g.has_lowner, g.has_lowner + BRDC_MAX_LEVELS, h->has_lowner);
    BRDC_CUDA(h, "brdc.graph_launch", cudaGraphLaunch(g.exec, h->stream));
    h->replayed = true;
    return BRDC_STATUS_SUCCESS;
}

// brdc_dstebr after its checks: a graph replay where graph_call takes the
// call, else the stream launches.
brdc_status plain_solve(brdc_handle h, const HostForest &hf, const Layout &L, const Forest &F,
                        const Ws &w, const double *D, const double *E, double *W, void *ws,
                        size_t ws_size, const double *srcD = nullptr,
                        const double *srcE = nullptr) {
    SolveSig sig;
    sig.kind = 0;
    sig.n = hf.total_n;
    sig.D = D;
    sig.E = E;
    sig.W = W;
    sig.ws = ws;
    sig.ws_size = ws_size;
    sig.srcD = srcD;
    sig.srcE = srcE;
    auto enqueue = [&]() { return run_forest(h, hf, L, F, w, D, E, W, srcD, srcE); };
    bool done = false;
    const brdc_status st = graph_call(h, h->gf, sig, enqueue, &done);
    return done ? st : enqueue();
}

} // namespace

// ------------------------------------------------------------------ C ABI

extern "C" const char *brdc_version(void) { return "brdc-b200 0.1"; }

extern "C" brdc_status brdc_create(brdc_handle *handle) {
    if (handle == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    *handle = nullptr;
    brdc_handle h = new (std::nothrow) brdc_handle_struct{};
    if (h == nullptr) {
        return BRDC_STATUS_ALLOC_FAILED;
    }
    h->prep_ws = nullptr;
    if (cudaGetDevice(&h->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount,
                               h->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) !=
            cudaSuccess) {
        delete h;
        return BRDC_STATUS_CUDA_ERROR;
    }
    h->stream = h->own_stream;
    *handle = h;
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_destroy(brdc_handle h) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (h->ev_ready) {
        for (auto &e : h->ev) {
            cudaEventDestroy(e);
        }
    }
    if (h->prep_ev != nullptr) {
        cudaEventDestroy(h->prep_ev);
    }
    drop_graph(h->gf);
    drop_graph(h->gb);
    if (h->gcap != nullptr) {
        cudaStreamDestroy(h->gcap);
    }
    if (h->own_stream != nullptr) {
        cudaStreamDestroy(h->own_stream);
    }
    delete h;
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_set_tuning(brdc_handle h, const brdc_tuning *t) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (t == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    const int c = t->deflate_cluster;
    if (t->subtree_levels < -1 || t->subtree_levels > kSubMaxLevels ||
        !(c == 1 || c == 2 || c == 4 || c == 8 || c == 16) || t->sweep_lanes_target < 1024 ||
        t->sweep_lanes_target > (1 << 24) || t->fused_level_rows < 0) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    h->sub_levels = t->subtree_levels;
    h->defl_cluster = c;
    h->lanes_target = t->sweep_lanes_target;
    h->lvl_rows = t->fused_level_rows;
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_set_limits(brdc_handle h, const brdc_limits *l) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (l == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    if (l->secular_max_iter < 1 || l->secular_max_iter > 1000 || l->wait_limit_ns < 0 ||
        l->wait_limit_ns > 1000000000000LL) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    h->max_iter = l->secular_max_iter;
    h->wait_ns = (unsigned long long)l->wait_limit_ns;
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_get_limits(brdc_handle h, brdc_limits *l) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (l == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    l->secular_max_iter = h->max_iter;
    l->reserved = 0;
    l->wait_limit_ns = (long long)h->wait_ns;
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_get_tuning(brdc_handle h, brdc_tuning *t) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (t == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    t->subtree_levels = h->sub_levels;
    t->deflate_cluster = h->defl_cluster;
    t->sweep_lanes_target = h->lanes_target;
    t->fused_level_rows = h->lvl_rows;
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_set_stream(brdc_handle h, brdc_stream_t stream) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    h->stream = reinterpret_cast<cudaStream_t>(stream);
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_get_stream(brdc_handle h, brdc_stream_t *stream) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (stream == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    *stream = reinterpret_cast<brdc_stream_t>(h->stream);
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_get_last_error(brdc_handle h, int *code,
                                           brdc_error_source *source,
                                           const char **site) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (code != nullptr) {
        *code = h->last_code;
    }
    if (source != nullptr) {
        *source = h->last_src;
    }
    if (site != nullptr) {
        *site = h->last_site;
    }
    return BRDC_STATUS_SUCCESS;
}

extern "C" const char *brdc_status_to_string(brdc_status status) {
    switch (status) {
    case BRDC_STATUS_SUCCESS: return "success";
    case BRDC_STATUS_INVALID_HANDLE: return "invalid_handle";
    case BRDC_STATUS_INVALID_POINTER: return "invalid_pointer";
    case BRDC_STATUS_INVALID_VALUE: return "invalid_value";
    case BRDC_STATUS_INVALID_WORKSPACE: return "invalid_workspace";
    case BRDC_STATUS_ALLOC_FAILED: return "alloc_failed";
    case BRDC_STATUS_CUDA_ERROR: return "cuda_error";
    case BRDC_STATUS_INTERNAL_ERROR: return "internal_error";
    case BRDC_STATUS_NOT_IMPLEMENTED: return "not_implemented";
    case BRDC_STATUS_NOT_CONVERGED: return "not_converged";
    default: return "unknown_status";
    }
}

extern "C" brdc_status brdc_dstebr_workspace_size(int64_t n, int flags,
                                                  size_t *bytes) {
    if (bytes == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    if (n <= 0 || n > (1LL << 30)) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    const long long off[2] = {0, (long long)n};
    HostForest f;
    if (!build_forest(1, off, &f)) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    *bytes = make_layout(f, (flags & BRDC_FLAG_KEEP_CHECKPOINTS) != 0).bytes;
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_dstebr(brdc_handle h, int64_t n, const double *d_D,
                                   const double *d_E, double *d_W,
                                   void *workspace, size_t workspace_size) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (d_D == nullptr || d_W == nullptr || (n > 1 && d_E == nullptr)) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    if (n <= 0 || n > (1LL << 30)) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    const long long off[2] = {0, (long long)n};
    HostForest hf;
    if (!build_forest(1, off, &hf)) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    // A workspace sized with BRDC_FLAG_KEEP_CHECKPOINTS records the
    // per-level state that brdc_dstebr_backward reads.
    const Layout Lc = make_layout(hf, true);
    const bool ckpt = workspace != nullptr && workspace_size >= Lc.bytes;
    const Layout L = ckpt ? Lc : make_layout(hf, false);
    if (workspace == nullptr || workspace_size < L.bytes) {
        return BRDC_STATUS_INVALID_WORKSPACE;
    }
    const Ws w = carve(workspace, hf, ckpt);
    Forest F{};
    F.B = 1;
    F.max_levels = hf.max_levels;
    F.n0 = n;
    F.L0 = hf.max_levels;
    return plain_solve(h, hf, L, F, w, d_D, d_E, d_W, workspace, workspace_size);
}

namespace {

// Workspace of brdc_dstebr_host: the plain solve's, then the device images
// [D | E] back to back (so that a host buffer holding E right after D is
// one copy) and W, each part 256-byte aligned.
struct HostLayout {
    size_t d, e, w, bytes;
};

HostLayout host_layout(long long n, const HostForest &hf) {
    HostLayout H;
    H.d = align_up(make_layout(hf, false).bytes);
    H.e = H.d + sizeof(double) * n;
    H.w = align_up(H.e + sizeof(double) * std::max(n - 1, 1LL));
    H.bytes = H.w + align_up(sizeof(double) * n);
    return H;
}

} // namespace

extern "C" brdc_status brdc_dstebr_host_workspace_size(int64_t n, size_t *bytes) {
    if (bytes == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    if (n <= 0 || n > (1LL << 30)) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    const long long off[2] = {0, (long long)n};
    HostForest hf;
    if (!build_forest(1, off, &hf)) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    *bytes = host_layout(n, hf).bytes;
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_dstebr_host(brdc_handle h, int64_t n, const double *h_D,
                                        const double *h_E, double *h_W, void *workspace,
                                        size_t workspace_size) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (h_D == nullptr || h_W == nullptr || (n > 1 && h_E == nullptr)) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    if (n <= 0 || n > (1LL << 30)) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    const long long off[2] = {0, (long long)n};
    HostForest hf;
    if (!build_forest(1, off, &hf)) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    const HostLayout H = host_layout(n, hf);
    if (workspace == nullptr || workspace_size < H.bytes) {
        return BRDC_STATUS_INVALID_WORKSPACE;
    }
    char *base = static_cast<char *>(workspace);
    double *dD = reinterpret_cast<double *>(base + H.d);
    double *dE = reinterpret_cast<double *>(base + H.e);
    double *dW = reinterpret_cast<double *>(base + H.w);
    const Layout L = make_layout(hf, false);
    const Ws w = carve(workspace, hf, false);
    Forest F{};
    F.B = 1;
    F.max_levels = hf.max_levels;
    F.n0 = n;
    F.L0 = hf.max_levels;
    // Page-locked D and E: k_norm reads them through their device addresses
    // and writes the device images as it takes the norm, so no copy in
    // precedes the solve (on B200, against the copies below: uniform 16,384
    // end to end 0.479 -> 0.473 ms, normal 65,536 0.678 -> 0.674 ms).
    // Otherwise the copies in on the stream.  Then the device entry's solve,
    // a graph replay from the second call with these buffers on.
    void *mD = nullptr, *mE = nullptr;
    if (cudaHostGetDevicePointer(&mD, const_cast<double *>(h_D), 0) != cudaSuccess ||
        (n > 1 && cudaHostGetDevicePointer(&mE, const_cast<double *>(h_E), 0) != cudaSuccess)) {
        cudaGetLastError();
        mD = mE = nullptr;
    }
    if (mD == nullptr) {
        // E right after D in the caller's memory: one copy of [D | E].  Two
        // separate page-locked allocations can also lie back to back, and the
        // runtime refuses a copy across them (an error it returns at once, with
        // nothing enqueued): then the two copies below.  Inside the caller's
        // stream capture a refused call would end the capture, so there the
        // copies are always two.
        bool joint = false;
        if (n > 1 && h_E == h_D + n) {
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusActive;
            if (cudaStreamIsCapturing(h->stream, &cs) == cudaSuccess &&
                cs == cudaStreamCaptureStatusNone) {
                joint = cudaMemcpyAsync(dD, h_D, sizeof(double) * (2 * n - 1),
                                        cudaMemcpyHostToDevice, h->stream) == cudaSuccess;
            }
            if (!joint) {
                cudaGetLastError();
            }
        }
        if (!joint) {
            BRDC_CUDA(h, "brdc.host.copy_d",
                      cudaMemcpyAsync(dD, h_D, sizeof(double) * n, cudaMemcpyHostToDevice,
                                      h->stream));
            if (n > 1) {
                BRDC_CUDA(h, "brdc.host.copy_e",
                          cudaMemcpyAsync(dE, h_E, sizeof(double) * (n - 1), cudaMemcpyHostToDevice,
                                          h->stream));
            }
        }
    }
    // W page-locked: the solve stores the eigenvalues through W's device
    // address straight into host memory as its last level places them, so
    // no copy out follows the solve (on B200, uniform 65,536 end to end
    // 0.776 -> 0.753 ms, 16,384 0.483 -> 0.477 ms, the medians of three
    // processes).  Otherwise they land in the device image and are copied.
    void *mW = nullptr;
    if (cudaHostGetDevicePointer(&mW, h_W, 0) != cudaSuccess) {
        cudaGetLastError();
        mW = nullptr;
    }
    double *Wd = mW != nullptr ? static_cast<double *>(mW) : dW;
    const double *sD = mD != nullptr ? static_cast<const double *>(mD) : nullptr;
    const double *sE = mD != nullptr ? (n > 1 ? static_cast<const double *>(mE) : sD) : nullptr;
    const brdc_status st = plain_solve(h, hf, L, F, w, dD, dE, Wd, workspace, workspace_size,
                                       sD, sE);
    if (st != BRDC_STATUS_SUCCESS || mW != nullptr) {
        return st;
    }
    BRDC_CUDA(h, "brdc.host.copy_w",
              cudaMemcpyAsync(h_W, dW, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    return BRDC_STATUS_SUCCESS;
}

namespace {
cudaError_t noalloc_cached_address(int device, void **out);
}

extern "C" brdc_status brdc_get_info(brdc_handle h, const void *workspace,
                                     int *info) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (workspace == nullptr || info == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    const WsHeader *hd = static_cast<const WsHeader *>(workspace);
    int vals[2] = {0, 0};
    BRDC_CUDA(h, "brdc.get_info.copy",
              cudaMemcpyAsync(vals, &hd->status, sizeof(int) * 2,
                              cudaMemcpyDeviceToHost, h->stream));
    BRDC_CUDA(h, "brdc.get_info.sync", cudaStreamSynchronize(h->stream));
    if (vals[0] != 0) {
        *info = -vals[0];
        set_error(h, vals[0], BRDC_ERROR_SRC_DEVICE, "brdc.device_status");
        return BRDC_STATUS_INTERNAL_ERROR;
    }
    *info = vals[1];
    return vals[1] > 0 ? BRDC_STATUS_NOT_CONVERGED : BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_get_diagnostics(brdc_handle h, const void *workspace,
                                            brdc_diagnostics *out) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (workspace == nullptr || out == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    WsHeader hd;
    BRDC_CUDA(h, "brdc.diagnostics.copy",
              cudaMemcpyAsync(&hd, workspace, sizeof(WsHeader),
                              cudaMemcpyDeviceToHost, h->stream));
    BRDC_CUDA(h, "brdc.diagnostics.sync", cudaStreamSynchronize(h->stream));
    std::memset(out, 0, sizeof(*out));
    out->n = (int)hd.total_n;
    out->levels = hd.max_levels;
    out->leaf_count = hd.leaf_count;
    out->leaf_sweeps_max = hd.leaf_sweeps_max;
    out->leaf_sweeps_sum = hd.leaf_sweeps_sum;
    for (int k = 0; k < hd.max_levels && k < BRDC_MAX_LEVELS; ++k) {
        out->level[k] = hd.diag[k];
        out->level[k].level = k;
        out->level[k].zero_deflated_total =
            hd.diag[k].size_sum - hd.diag[k].dd_before_sum;
        out->level[k].close_deflated_total =
            hd.diag[k].dd_before_sum - hd.diag[k].dd_after_sum;
    }
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_get_merge_trace(brdc_handle h, const void *workspace,
                                            size_t workspace_size, int64_t n, int level,
                                            double *d, double *z, int *row, int *state,
                                            int *link, double *c, double *s, int *node_K,
                                            double *node_rho, double *node_tol) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (workspace == nullptr || d == nullptr || z == nullptr || row == nullptr ||
        state == nullptr || link == nullptr || c == nullptr || s == nullptr ||
        node_K == nullptr || node_rho == nullptr || node_tol == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    const long long off[2] = {0, (long long)n};
    HostForest hf;
    if (n <= 0 || n > (1LL << 30) || !build_forest(1, off, &hf) || level < 0 ||
        level >= hf.max_levels) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    const Layout L = make_layout(hf, true);
    if (workspace_size < L.bytes) {
        return BRDC_STATUS_INVALID_WORKSPACE;
    }
    Ws w = carve(const_cast<void *>(workspace), hf, true);
    level_view(hf, L, w, level, &w);
    const int depth = hf.max_levels - 1 - level;
    const int nodes = 1 << depth;
    std::vector<double> md(n), mz(n), gc(n), gsn(n);
    std::vector<int> morig(n), amap(n), gmark(n), gbase(n), zmap(n), pmap(L.np), nK(nodes), nKz(nodes);
    std::vector<double> nrho(nodes), ntol(nodes);
    auto get = [&](void *dst, const void *src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream);
    };
    const size_t nd = sizeof(double) * (size_t)n, ni = sizeof(int) * (size_t)n;
    cudaError_t e = cudaSuccess;
    e = e != cudaSuccess ? e : get(md.data(), w.md, nd);
    e = e != cudaSuccess ? e : get(mz.data(), w.mz, nd);
    e = e != cudaSuccess ? e : get(gc.data(), w.gc, nd);
    e = e != cudaSuccess ? e : get(gsn.data(), w.gs, nd);
    e = e != cudaSuccess ? e : get(morig.data(), w.morig, ni);
    e = e != cudaSuccess ? e : get(amap.data(), w.amap, ni);
    e = e != cudaSuccess ? e : get(gmark.data(), w.gmark, ni);
    e = e != cudaSuccess ? e : get(gbase.data(), w.gbase, ni);
    e = e != cudaSuccess ? e : get(zmap.data(), w.zmap, ni);
    e = e != cudaSuccess ? e : get(pmap.data(), w.pmap, sizeof(int) * (size_t)L.np);
    e = e != cudaSuccess ? e : get(nK.data(), w.nK, sizeof(int) * nodes);
    e = e != cudaSuccess ? e : get(nKz.data(), w.nKz, sizeof(int) * nodes);
    e = e != cudaSuccess ? e : get(nrho.data(), w.nrho, sizeof(double) * nodes);
    e = e != cudaSuccess ? e : get(ntol.data(), w.ntol, sizeof(double) * nodes);
    BRDC_CUDA(h, "brdc.merge_trace.copy", e);
    BRDC_CUDA(h, "brdc.merge_trace.sync", cudaStreamSynchronize(h->stream));
    for (int g = 0; g < nodes; ++g) {
        long long gs = 0, m = 0;
        walk_node(n, depth, g, &gs, &m);
        const long long po = (gs + g + 1) & ~1LL;
        const int K = nK[g], Kz = nKz[g];
        if (K < 0 || Kz < K || Kz > m) {
            set_error(h, 0, BRDC_ERROR_SRC_NONE, "brdc.merge_trace: no checkpoint of this level");
            return BRDC_STATUS_INVALID_VALUE;
        }
        node_K[g] = K;
        node_rho[g] = nrho[g];
        node_tol[g] = ntol[g];
        std::vector<int> pole_of_active(Kz, -1);
        for (int j = 0; j < K; ++j) {
            const int a = pmap[po + j];
            if (a >= 0 && a < Kz) {
                pole_of_active[a] = j;
            }
        }
        for (long long p = 0; p < m; ++p) {
            d[gs + p] = md[gs + p];
            z[gs + p] = mz[gs + p];
            row[gs + p] = morig[gs + p];
            state[gs + p] = -1;
            link[gs + p] = -1;
            c[gs + p] = 0.0;
            s[gs + p] = 0.0;
        }
        for (int a = 0; a < Kz; ++a) {
            const long long p = gs + amap[gs + a];
            if (gmark[gs + a]) {
                state[p] = 2;
                link[p] = amap[gs + gbase[gs + a]];
                c[p] = gc[gs + a];
                s[p] = gsn[gs + a];
            } else {
                state[p] = 0;
                link[p] = pole_of_active[a];
            }
        }
        for (long long q = 0; q < m - Kz; ++q) {
            state[gs + zmap[gs + q]] = 1;
        }
    }
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_set_timing(brdc_handle h, int enable) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (enable && !h->ev_ready) {
        for (auto &e : h->ev) {
            BRDC_CUDA(h, "brdc.timing.event_create", cudaEventCreate(&e));
        }
        h->ev_ready = 1;
    }
    h->timing = enable ? 1 : 0;
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_set_graphs(brdc_handle h, int enable) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    h->graphs = enable ? 1 : 0;
    if (!h->graphs) {
        for (SolveGraph *g : {&h->gf, &h->gb}) {
            drop_graph(*g);
            g->seen_valid = false;
        }
    }
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_get_last_launches(brdc_handle h, int *launches, int *replayed) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (launches == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    if (replayed != nullptr) {
        *replayed = h->replayed ? 1 : 0;
    }
    *launches = h->launches;
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_get_last_timings(brdc_handle h, brdc_timings *out) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (out == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    std::memset(out, 0, sizeof(*out));
    if (!h->timing || !h->ev_ready || h->ev_used < 3) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    BRDC_CUDA(h, "brdc.timing.sync", cudaStreamSynchronize(h->stream));
    auto el = [&](int a, int b) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, h->ev[a], h->ev[b]);
        return ms;
    };
    out->init_ms = el(0, 1);
    out->leaf_ms = el(1, 2);
    out->levels = h->timed_levels;
    out->launches = h->launches;
    out->fused_levels = h->fused_levels;
    int prev = 2;
    for (int k = h->fused_levels; k < h->timed_levels; ++k) {
        const float m = el(prev, 3 + 4 * k);
        const float s = el(3 + 4 * k, 4 + 4 * k);
        const float l = el(4 + 4 * k, 5 + 4 * k);
        const float r = el(5 + 4 * k, 6 + 4 * k);
        out->level_ms[k][0] = m;
        out->level_ms[k][1] = s;
        out->level_ms[k][2] = l;
        out->level_ms[k][3] = r;
        out->merge_ms += m;
        out->secular_ms += s;
        out->lowner_ms += l;
        out->rows_ms += r;
        prev = 6 + 4 * k;
    }
    out->total_ms = el(0, prev);
    return BRDC_STATUS_SUCCESS;
}

// --------------------------------------------------------------- batched

namespace {

// Forest descriptor of a batch.  With more than one instance the
// per-instance tables (row offsets, levels, node, leaf and subtree
// prefixes) live in the workspace.  Every call outside a stream capture
// writes them, because anything may have reused the workspace since the
// last batched call (a single solve carves the same bytes differently, and
// a caching allocator hands addresses back).  A captured call writes none,
// so the graph replays only kernels: it needs the last non-captured batched
// call of this handle to have written the tables for the same workspace,
// offsets and layout, and the workspace to stay reserved for the graph.
brdc_status prepare_forest(brdc_handle h, const HostForest &hf, const Ws &w,
                           const void *workspace, bool ckpt, Forest *F) {
    *F = Forest{};
    F->B = hf.B;
    F->max_levels = hf.max_levels;
    if (hf.B == 1) {
        F->n0 = hf.total_n;
        F->L0 = hf.max_levels;
        return BRDC_STATUS_SUCCESS;
    }
    const int sub = effective_sub_levels(h, hf);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    BRDC_CUDA(h, "brdc.batched.capture_status", cudaStreamIsCapturing(h->stream, &cap));
    if (cap != cudaStreamCaptureStatusNone) {
        const bool same = h->prep_ws == workspace && h->prep_ckpt == ckpt &&
                          h->prep_sub == sub && h->prep_off.size() == (size_t)hf.B + 1 &&
                          std::equal(h->prep_off.begin(), h->prep_off.end(), hf.off.begin());
        if (!same) {
            set_error(h, 0, BRDC_ERROR_SRC_NONE,
                      "brdc.batched: a captured call needs a non-captured call with the "
                      "same workspace and offsets first");
            return BRDC_STATUS_INVALID_VALUE;
        }
    } else {
        // the host tables of the previous upload stay alive until its copies ran
        if (h->prep_ev == nullptr) {
            BRDC_CUDA(h, "brdc.batched.event_create",
                      cudaEventCreateWithFlags(&h->prep_ev, cudaEventDisableTiming));
        }
        if (h->prep_pending) {
            BRDC_CUDA(h, "brdc.batched.event_wait", cudaEventSynchronize(h->prep_ev));
            h->prep_pending = false;
        }
        const size_t B1 = (size_t)hf.B + 1;
        const size_t Lm = (size_t)std::max(hf.max_levels, 1);
        // [lev (B) | node prefixes (B+1 per level) | leaf prefix (B+1) | subtree prefix (B+1)]
        std::vector<int> &tab = h->prep_tab;
        tab.assign((size_t)hf.B + B1 * Lm + 2 * B1, 0);
        int *lev = tab.data();
        int *node_prefix = lev + hf.B;
        int *leaf_prefix = node_prefix + B1 * Lm;
        int *sub_prefix = leaf_prefix + B1;
        for (int b = 0; b < hf.B; ++b) {
            lev[b] = hf.lev[b];
        }
        for (int k = 0; k < hf.max_levels; ++k) {
            int *row = node_prefix + (size_t)k * B1;
            for (int b = 0; b < hf.B; ++b) {
                const int L = hf.lev[b];
                row[b + 1] = row[b] + (L > k ? (1 << (L - 1 - k)) : 0);
            }
        }
        for (int b = 0; b < hf.B; ++b) {
            leaf_prefix[b + 1] = leaf_prefix[b] + (1 << hf.lev[b]);
            sub_prefix[b + 1] = sub_prefix[b] + (int)subtrees_of(hf.lev[b], sub);
        }
        h->prep_off = hf.off;
        BRDC_CUDA(h, "brdc.batched.upload_off",
                  cudaMemcpyAsync(w.f_off, h->prep_off.data(), sizeof(long long) * B1,
                                  cudaMemcpyHostToDevice, h->stream));
        BRDC_CUDA(h, "brdc.batched.upload_lev",
                  cudaMemcpyAsync(w.f_lev, lev, sizeof(int) * hf.B, cudaMemcpyHostToDevice,
                                  h->stream));
        BRDC_CUDA(h, "brdc.batched.upload_nodes",
                  cudaMemcpyAsync(w.f_node_prefix, node_prefix, sizeof(int) * B1 * Lm,
                                  cudaMemcpyHostToDevice, h->stream));
        BRDC_CUDA(h, "brdc.batched.upload_leaves",
                  cudaMemcpyAsync(w.f_leaf_prefix, leaf_prefix, sizeof(int) * B1,
                                  cudaMemcpyHostToDevice, h->stream));
        BRDC_CUDA(h, "brdc.batched.upload_subtrees",
                  cudaMemcpyAsync(w.f_sub_prefix, sub_prefix, sizeof(int) * B1,
                                  cudaMemcpyHostToDevice, h->stream));
        BRDC_CUDA(h, "brdc.batched.upload_record", cudaEventRecord(h->prep_ev, h->stream));
        h->prep_pending = true;
        h->prep_ws = workspace;
        h->prep_ckpt = ckpt;
        h->prep_sub = sub;
    }
    F->off = w.f_off;
    F->lev = w.f_lev;
    F->node_prefix = w.f_node_prefix;
    F->leaf_prefix = w.f_leaf_prefix;
    F->sub_prefix = w.f_sub_prefix;
    return BRDC_STATUS_SUCCESS;
}

brdc_status batch_forest(int64_t count, const int64_t *offsets, HostForest *hf) {
    if (offsets == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    if (count <= 0 || count > (1LL << 28) || offsets[0] != 0) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    if (!build_forest((int)count, reinterpret_cast<const long long *>(offsets), hf)) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    return BRDC_STATUS_SUCCESS;
}

} // namespace

extern "C" brdc_status brdc_dstebr_batched_workspace_size(int64_t count,
                                                          const int64_t *offsets,
                                                          size_t *bytes) {
    if (bytes == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    HostForest f;
    const brdc_status st = batch_forest(count, offsets, &f);
    if (st != BRDC_STATUS_SUCCESS) {
        return st;
    }
    *bytes = make_layout(f).bytes;
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_dstebr_batched_checkpoint_workspace_size(int64_t count,
                                                                     const int64_t *offsets,
                                                                     size_t *bytes) {
    if (bytes == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    HostForest f;
    const brdc_status st = batch_forest(count, offsets, &f);
    if (st != BRDC_STATUS_SUCCESS) {
        return st;
    }
    *bytes = make_layout(f, true).bytes;
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_dstebr_batched(brdc_handle h, int64_t count,
                                           const int64_t *offsets,
                                           const double *d_D, const double *d_E,
                                           double *d_W, void *workspace,
                                           size_t workspace_size) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (d_D == nullptr || d_W == nullptr || d_E == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    HostForest hf;
    brdc_status st = batch_forest(count, offsets, &hf);
    if (st != BRDC_STATUS_SUCCESS) {
        return st;
    }
    // a workspace of the checkpoint size records what the backward reads
    const Layout Lc = make_layout(hf, true);
    const bool ckpt = workspace != nullptr && workspace_size >= Lc.bytes;
    const Layout L = ckpt ? Lc : make_layout(hf, false);
    if (workspace == nullptr || workspace_size < L.bytes) {
        return BRDC_STATUS_INVALID_WORKSPACE;
    }
    const Ws w = carve(workspace, hf, ckpt);
    Forest F;
    st = prepare_forest(h, hf, w, workspace, ckpt, &F);
    if (st != BRDC_STATUS_SUCCESS) {
        return st;
    }
    return run_forest(h, hf, L, F, w, d_D, d_E, d_W);
}

// ------------------------------------------------------------- autotuner

extern "C" brdc_status brdc_autotune(brdc_handle h, int64_t count, const int64_t *offsets,
                                     const double *d_D, const double *d_E, double *d_W,
                                     void *workspace, size_t workspace_size,
                                     brdc_tuning *best) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    HostForest hf;
    brdc_status st = batch_forest(count, offsets, &hf);
    if (st != BRDC_STATUS_SUCCESS) {
        return st;
    }
    cudaEvent_t e0, e1;
    BRDC_CUDA(h, "brdc.autotune.event", cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        set_error(h, (int)cudaErrorMemoryAllocation, BRDC_ERROR_SRC_CUDA, "brdc.autotune.event");
        return BRDC_STATUS_CUDA_ERROR;
    }
    const brdc_tuning saved{h->sub_levels, h->defl_cluster, h->lanes_target, h->lvl_rows};
    brdc_tuning cur{effective_sub_levels(h, hf), h->defl_cluster, h->lanes_target, h->lvl_rows};
    int reps = 3;
    // median device time of a few solves under tuning t (first call warms
    // up and, for a new subtree depth, uploads the batch tables)
    auto run = [&](const brdc_tuning &t, float *ms) -> brdc_status {
        h->sub_levels = t.subtree_levels;
        h->defl_cluster = t.deflate_cluster;
        h->lanes_target = t.sweep_lanes_target;
        h->lvl_rows = t.fused_level_rows;
        brdc_status r = brdc_dstebr_batched(h, count, offsets, d_D, d_E, d_W, workspace,
                                            workspace_size);
        if (r != BRDC_STATUS_SUCCESS) {
            return r;
        }
        float v[5];
        for (int i = 0; i < reps; ++i) {
            cudaEventRecord(e0, h->stream);
            r = brdc_dstebr_batched(h, count, offsets, d_D, d_E, d_W, workspace, workspace_size);
            cudaEventRecord(e1, h->stream);
            if (r != BRDC_STATUS_SUCCESS) {
                return r;
            }
            BRDC_CUDA(h, "brdc.autotune.sync", cudaEventSynchronize(e1));
            cudaEventElapsedTime(&v[i], e0, e1);
        }
        std::sort(v, v + reps);
        *ms = v[reps / 2];
        return BRDC_STATUS_SUCCESS;
    };
    float best_ms = 0.0f;
    st = run(cur, &best_ms);
    if (st == BRDC_STATUS_SUCCESS && best_ms > 50.0f) {
        reps = 1; // long solves: one timed run per candidate
    }
    // coordinate descent, one parameter at a time: subtree depth, fused
    // levels, deflation cluster, sweep lanes
    const int subs[] = {0, 1, 2, 3, 4, 5};
    const int fuse[] = {0, kLvlRowsPerCta, 1 << 30};
    const int clusters[] = {1, 2, 4, 8, 16};
    const int lanes[] = {37888, 75776, 151552, 303104, 606208};
    struct Axis {
        int brdc_tuning::*field;
        const int *vals;
        int nv;
    };
    const Axis axes[] = {{&brdc_tuning::subtree_levels, subs, 6},
                         {&brdc_tuning::fused_level_rows, fuse, 3},
                         {&brdc_tuning::deflate_cluster, clusters, 5},
                         {&brdc_tuning::sweep_lanes_target, lanes, 5}};
    const int mmax_all = *std::max_element(hf.level_mmax.begin(), hf.level_mmax.end());
    for (const Axis &ax : axes) {
        if (st != BRDC_STATUS_SUCCESS) {
            break;
        }
        if (ax.field == &brdc_tuning::deflate_cluster && mmax_all < 2 * kDeflEPT * 1024) {
            continue; // no merge is large enough for a cluster
        }
        brdc_tuning pick = cur;
        for (int i = 0; i < ax.nv && st == BRDC_STATUS_SUCCESS; ++i) {
            brdc_tuning t = cur;
            if (t.*ax.field == ax.vals[i]) {
                continue;
            }
            t.*ax.field = ax.vals[i];
            float ms = 0.0f;
            st = run(t, &ms);
            if (st == BRDC_STATUS_SUCCESS && ms < best_ms) {
                best_ms = ms;
                pick = t;
            }
        }
        cur = pick;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != BRDC_STATUS_SUCCESS) {
        h->sub_levels = saved.subtree_levels;
        h->defl_cluster = saved.deflate_cluster;
        h->lanes_target = saved.sweep_lanes_target;
        h->lvl_rows = saved.fused_level_rows;
        return st;
    }
    h->sub_levels = cur.subtree_levels;
    h->defl_cluster = cur.deflate_cluster;
    h->lanes_target = cur.sweep_lanes_target;
    h->lvl_rows = cur.fused_level_rows;
    if (best != nullptr) {
        *best = cur;
    }
    return BRDC_STATUS_SUCCESS;
}

// -------------------------------------------------------------- backward
namespace {

// Every adjoint kernel starts with pdl_begin, so each is launched with the
// programmatic-serialization attribute: its blocks are scheduled while the
// kernel before it finishes, and they wait there for its writes.
template <typename... P, typename... A>
void launch_pdl(void (*kern)(P...), long long grid, unsigned block, cudaStream_t s, A... args) {
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = plain_config((unsigned)grid, block, 0, s, at);
    cudaLaunchKernelEx(&cfg, kern, args...);
}

template <int T>
void launch_undeflate(const BArgs &b, int grid, cudaStream_t s) {
    launch_pdl(k_bw_undeflate<T>, grid, T, s, b);
}

void launch_undeflate_sized(const BArgs &b, int mmax, cudaStream_t s) {
    int t = 32;
    while (t < 1024 && t * 4 < mmax) {
        t <<= 1;
    }
    switch (t) {
    case 32: launch_undeflate<32>(b, b.nodes, s); break;
    case 64: launch_undeflate<64>(b, b.nodes, s); break;
    case 128: launch_undeflate<128>(b, b.nodes, s); break;
    case 256: launch_undeflate<256>(b, b.nodes, s); break;
    case 512: launch_undeflate<512>(b, b.nodes, s); break;
    default: launch_undeflate<1024>(b, b.nodes, s); break;
    }
}

// Reverse pass over a workspace holding the forward solve's checkpoints.
brdc_status run_backward(brdc_handle h, const HostForest &hf, const Layout &L,
                         const Forest &F, const Ws &w, const double *D,
                         const double *E, const double *G, double *gD, double *gE) {
    cudaStream_t s = h->stream;
    const long long nt = hf.total_n;
    long long eg = (nt + 255) / 256;
    eg = std::max<long long>(1, std::min<long long>(eg, (long long)h->sm_count * 8));
    // E holds n-1 entries for one instance, one per row (the last of each
    // instance unused and returned as 0) for a batch
    const long long ne = hf.B > 1 ? nt : nt - 1;
    if (ne > 0) {
        launch_pdl(k_bw_zero, eg, 256, s, gE, ne);
        BRDC_CUDA(h, "brdc.bw.zero_ge", cudaGetLastError());
    }
    double *par[3] = {w.bnd, w.bnf, w.bnl};
    double *out[3] = {w.bcd, w.bcf, w.bcl};
    // k_bw_roots and k_bw_poles: 64 registers or fewer, four blocks per SM
    const int wgrid = h->sm_count * 4;
    long long dgrid = (4 * nt + 255) / 256;
    dgrid = std::max<long long>(1, std::min<long long>(dgrid, (long long)h->sm_count * 16));
    for (int k = hf.max_levels - 1; k >= 0; --k) {
        Ws wl = w;
        level_view(hf, L, w, k, &wl);
        wl.bnd = par[0];
        wl.bnf = par[1];
        wl.bnl = par[2];
        wl.bcd = out[0];
        wl.bcf = out[1];
        wl.bcl = out[2];
        BArgs b{};
        b.F = F;
        b.w = wl;
        b.D = D;
        b.E = E;
        b.G = G;
        b.gD = gD;
        b.gE = gE;
        b.k = k;
        b.nodes = hf.level_nodes[k];
        b.level_rows = hf.level_rows[k];
        b.lanes_target = h->lanes_target;
        launch_pdl(k_bw_unplace, eg, 256, s, b, nt);
        launch_pdl(k_bw_roots, wgrid, kSweepThreads, s, b);
        launch_pdl(k_bw_poles, wgrid, kSweepThreads, s, b);
        if (k + 1 < hf.max_levels || hf.B > 1) {
            // up to 4 lanes per row (the kernel picks); surplus blocks exit
            launch_pdl(k_bw_defl, dgrid, 256, s, b, nt);
        }
        if (hf.level_mmax[k] >= 2 * kDeflEPT * 1024) {
            // large merges: grid-wide passes instead of one CTA per merge
            launch_pdl(k_bw_ud_active, eg, 256, s, b, nt);
            launch_pdl(k_bw_ud_chains, eg, 256, s, b, nt);
            launch_pdl(k_bw_ud_merged, eg, 256, s, b, nt);
            launch_pdl(k_bw_ud_children, eg, 256, s, b, nt);
            launch_pdl(k_bw_ud_rho, std::max(1, std::min(b.nodes / 8 + 1, h->sm_count * 8)), 256, s, b);
        } else {
            launch_undeflate_sized(b, hf.level_mmax[k], s);
        }
        BRDC_CUDA(h, "brdc.bw.level", cudaGetLastError());
        std::swap(par[0], out[0]);
        std::swap(par[1], out[1]);
        std::swap(par[2], out[2]);
    }
    Ws wl = w;
    wl.bcd = par[0];
    wl.bcf = par[1];
    wl.bcl = par[2];
    BArgs b{};
    b.F = F;
    b.w = wl;
    b.D = D;
    b.E = E;
    b.G = G;
    b.gD = gD;
    b.gE = gE;
    const long long per = 2LL * kLeafWarps;
    long long grid = (hf.leaves + per - 1) / per;
    grid = std::max<long long>(1, std::min<long long>(grid, (long long)h->sm_count * 16));
    launch_pdl(k_bw_leaf, grid, kLeafWarps * 32, s, b, hf.leaves);
    BRDC_CUDA(h, "brdc.bw.leaf", cudaGetLastError());
    long long cg = (hf.leaves + 255) / 256;
    cg = std::max<long long>(1, std::min<long long>(cg, (long long)h->sm_count * 8));
    launch_pdl(k_bw_cuts, cg, 256, s, b, hf.leaves);
    BRDC_CUDA(h, "brdc.bw.cuts", cudaGetLastError());
    return BRDC_STATUS_SUCCESS;
}

} // namespace

extern "C" brdc_status brdc_dstebr_backward(brdc_handle h, int64_t n,
                                            const double *d_D, const double *d_E,
                                            const double *d_G, double *d_gD,
                                            double *d_gE, void *workspace,
                                            size_t workspace_size,
                                            int keep_forward) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (d_D == nullptr || d_G == nullptr || d_gD == nullptr ||
        (n > 1 && (d_E == nullptr || d_gE == nullptr))) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    if (n <= 0 || n > (1LL << 30)) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    const long long off[2] = {0, (long long)n};
    HostForest hf;
    if (!build_forest(1, off, &hf)) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    const Layout L = make_layout(hf, true);
    if (workspace == nullptr || workspace_size < L.bytes) {
        return BRDC_STATUS_INVALID_WORKSPACE;
    }
    const Ws w = carve(workspace, hf, true);
    Forest F{};
    F.B = 1;
    F.max_levels = hf.max_levels;
    F.n0 = n;
    F.L0 = hf.max_levels;
    auto enqueue = [&]() {
        if (!keep_forward) {
            const brdc_status st = run_forest(h, hf, L, F, w, d_D, d_E, w.wtmp);
            if (st != BRDC_STATUS_SUCCESS) {
                return st;
            }
        }
        return run_backward(h, hf, L, F, w, d_D, d_E, d_G, d_gD, d_gE);
    };
    SolveSig sig;
    sig.kind = 1;
    sig.n = n;
    sig.D = d_D;
    sig.E = d_E;
    sig.ws = workspace;
    sig.ws_size = workspace_size;
    sig.G = d_G;
    sig.gD = d_gD;
    sig.gE = d_gE;
    sig.keep_forward = keep_forward ? 1 : 0;
    bool done = false;
    const brdc_status st = graph_call(h, h->gb, sig, enqueue, &done);
    return done ? st : enqueue();
}

extern "C" brdc_status brdc_dstebr_batched_backward(brdc_handle h, int64_t count,
                                                    const int64_t *offsets,
                                                    const double *d_D, const double *d_E,
                                                    const double *d_G, double *d_gD,
                                                    double *d_gE, void *workspace,
                                                    size_t workspace_size,
                                                    int keep_forward) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (d_D == nullptr || d_E == nullptr || d_G == nullptr || d_gD == nullptr ||
        d_gE == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    HostForest hf;
    brdc_status st = batch_forest(count, offsets, &hf);
    if (st != BRDC_STATUS_SUCCESS) {
        return st;
    }
    const Layout L = make_layout(hf, true);
    if (workspace == nullptr || workspace_size < L.bytes) {
        return BRDC_STATUS_INVALID_WORKSPACE;
    }
    const Ws w = carve(workspace, hf, true);
    Forest F;
    st = prepare_forest(h, hf, w, workspace, true, &F);
    if (st != BRDC_STATUS_SUCCESS) {
        return st;
    }
    if (!keep_forward) {
        st = run_forest(h, hf, L, F, w, d_D, d_E, w.wtmp);
        if (st != BRDC_STATUS_SUCCESS) {
            return st;
        }
    }
    return run_backward(h, hf, L, F, w, d_D, d_E, d_G, d_gD, d_gE);
}

// ------------------------------------------------- LAPACK-style host entry
namespace {
int wprod_nthreads_host() {
    // BRDC_WPROD_NTHREADS (cpu/src/dstedc_dc_br.f:153-213) with the team
    // size taken from OMP_NUM_THREADS (1 when unset).
    int nt = 1;
    if (const char *s = std::getenv("OMP_NUM_THREADS")) {
        nt = std::max(1, std::atoi(s));
    }
    int val = 0;
    if (const char *s = std::getenv("OPENBLAS_BRDC_WPROD_THREADS")) {
        for (const char *p = s; *p != '\0' && p - s < 32; ++p) {
            if (*p >= '0' && *p <= '9') {
                val = 10 * val + (*p - '0');
            } else if (*p != ' ') {
                val = 0;
                break;
            }
        }
    }
    if (val > 0) {
        return std::max(1, std::min(val, nt));
    }
    const int cap = nt <= 1 ? 1 : nt <= 8 ? 2 : nt <= 28 ? 4 : 16;
    return std::max(1, std::min(cap, nt));
}
} // namespace

namespace {

// Argument checks and workspace query of DSTEDC_DC_BR
// (cpu/src/dstedc_dc_br.f:44-75): LWMIN = max(1,(16+2*NTHR)*N) and
// LIWMIN = max(1,7*N) above the LAPACK crossover (ILAENV(9) = 25), else 1;
// INFO = -1/-5/-7 for a bad N/LWORK/LIWORK; LWORK = -1 or LIWORK = -1 is a
// query.  Returns true when the caller goes on to solve.
bool stebr_check(int n, int lwork, int liwork, int *lwmin, int *liwmin, int *info) {
    *info = 0;
    *lwmin = 1;
    *liwmin = 1;
    const bool lquery = (lwork == -1 || liwork == -1);
    if (n < 0) {
        *info = -1;
        return false;
    }
    const int smlsiz = 25; // ILAENV(9, 'DSTEDC', ...)
    if (n > smlsiz) {
        *lwmin = std::max(1, (16 + 2 * wprod_nthreads_host()) * n);
        *liwmin = std::max(1, 7 * n);
    }
    if (lwork < *lwmin && !lquery) {
        *info = -5;
    } else if (liwork < *liwmin && !lquery) {
        *info = -7;
    }
    return !(*info != 0 || lquery || n == 0 || n == 1);
}

// The GPU solve behind the LAPACK-style entries: host D[n] and E[n-1] in,
// ascending eigenvalues out in D.  Allocates its device buffers (the caller
// passes host arrays) and synchronises.  Returns 0, the INFO > 0 of a root
// that did not converge, or n + 1 when the device could not be used.
int host_stebr(int n, double *d, const double *e) {
    brdc_handle h = nullptr;
    if (brdc_create(&h) != BRDC_STATUS_SUCCESS) {
        return n + 1;
    }
    size_t ws_bytes = 0;
    brdc_dstebr_workspace_size(n, 0, &ws_bytes);
    double *dD = nullptr, *dE = nullptr, *dW = nullptr;
    void *ws = nullptr;
    int fail = 0;
    fail |= cudaMalloc(&dD, sizeof(double) * n) != cudaSuccess;
    fail |= cudaMalloc(&dE, sizeof(double) * std::max(n - 1, 1)) != cudaSuccess;
    fail |= cudaMalloc(&dW, sizeof(double) * n) != cudaSuccess;
    fail |= cudaMalloc(&ws, ws_bytes) != cudaSuccess;
    if (!fail) {
        fail |= cudaMemcpyAsync(dD, d, sizeof(double) * n, cudaMemcpyHostToDevice,
                                h->stream) != cudaSuccess;
        fail |= cudaMemcpyAsync(dE, e, sizeof(double) * (n - 1),
                                cudaMemcpyHostToDevice, h->stream) != cudaSuccess;
    }
    int dinfo = 0;
    if (!fail) {
        fail |= brdc_dstebr(h, n, dD, dE, dW, ws, ws_bytes) != BRDC_STATUS_SUCCESS;
    }
    if (!fail) {
        const brdc_status st = brdc_get_info(h, ws, &dinfo);
        fail |= !(st == BRDC_STATUS_SUCCESS || st == BRDC_STATUS_NOT_CONVERGED);
    }
    if (!fail) {
        fail |= cudaMemcpyAsync(d, dW, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                h->stream) != cudaSuccess;
        fail |= cudaStreamSynchronize(h->stream) != cudaSuccess;
    }
    cudaFree(dD);
    cudaFree(dE);
    cudaFree(dW);
    cudaFree(ws);
    brdc_destroy(h);
    return fail ? n + 1 : (dinfo > 0 ? dinfo : 0);
}

} // namespace

extern "C" void brdc_dstedc_dc_br_(const int *n_, double *d, double *e,
                                   double *work, const int *lwork_,
                                   int *iwork, const int *liwork_, int *info) {
    const int n = *n_;
    int lwmin = 1, liwmin = 1;
    const bool go = stebr_check(n, *lwork_, *liwork_, &lwmin, &liwmin, info);
    if (*info == -1) {
        return;
    }
    work[0] = (double)lwmin;
    iwork[0] = liwmin;
    if (!go) {
        return;
    }
    const int r = host_stebr(n, d, e);
    if (r != 0) {
        *info = r;
    }
    work[0] = (double)lwmin;
    iwork[0] = liwmin;
}

// The BR routine under its upstream LAPACK name (README.md:13): the
// argument list and semantics of DSTEDC_DC_BR.
extern "C" void dstebr_(const int *n, double *d, double *e, double *work, const int *lwork,
                        int *iwork, const int *liwork, int *info) {
    brdc_dstedc_dc_br_(n, d, e, work, lwork, iwork, liwork, info);
}

// Single precision: the same checks and query (LWMIN counted in reals); the
// solve runs in FP64 on the GPU and the eigenvalues are rounded to float.
extern "C" void sstebr_(const int *n_, float *d, float *e, float *work, const int *lwork_,
                        int *iwork, const int *liwork_, int *info) {
    const int n = *n_;
    int lwmin = 1, liwmin = 1;
    const bool go = stebr_check(n, *lwork_, *liwork_, &lwmin, &liwmin, info);
    if (*info == -1) {
        return;
    }
    work[0] = (float)lwmin;
    iwork[0] = liwmin;
    if (!go) {
        return;
    }
    std::vector<double> dd(d, d + n), ee(e, e + (n - 1));
    const int r = host_stebr(n, dd.data(), ee.data());
    if (r != 0) {
        *info = r;
    }
    if (r <= n) { // solved (possibly with a root that hit the cap)
        for (int i = 0; i < n; ++i) {
            d[i] = (float)dd[i];
        }
    }
    work[0] = (float)lwmin;
    iwork[0] = liwmin;
}

// LAPACKE-style C wrappers (the upstream routine ships them too): the
// _work form passes the caller's workspace through, the plain form checks
// D and E for NaN (-2, -3), queries and allocates the workspace itself
// (LAPACK_WORK_MEMORY_ERROR = -1010 when that fails).
extern "C" int LAPACKE_dstebr_work(int n, double *d, double *e, double *work, int lwork,
                                   int *iwork, int liwork) {
    int info = 0;
    dstebr_(&n, d, e, work, &lwork, iwork, &liwork, &info);
    return info;
}

extern "C" int LAPACKE_sstebr_work(int n, float *d, float *e, float *work, int lwork,
                                   int *iwork, int liwork) {
    int info = 0;
    sstebr_(&n, d, e, work, &lwork, iwork, &liwork, &info);
    return info;
}

namespace {

template <typename R, typename Work>
int lapacke_stebr(int n, R *d, R *e, Work call) {
    if (n < 0) {
        return -1;
    }
    for (int i = 0; i < n; ++i) {
        if (d[i] != d[i]) {
            return -2;
        }
    }
    for (int i = 0; i + 1 < n; ++i) {
        if (e[i] != e[i]) {
            return -3;
        }
    }
    R wq = 0;
    int iwq = 0;
    int info = call(n, d, e, &wq, -1, &iwq, -1);
    if (info != 0) {
        return info;
    }
    const int lwork = std::max(1, (int)wq), liwork = std::max(1, iwq);
    std::vector<R> work;
    std::vector<int> iwork;
    try {
        work.resize((size_t)lwork);
        iwork.resize((size_t)liwork);
    } catch (...) {
        return -1010;
    }
    return call(n, d, e, work.data(), lwork, iwork.data(), liwork);
}

} // namespace

extern "C" int LAPACKE_dstebr(int n, double *d, double *e) {
    return lapacke_stebr<double>(n, d, e, LAPACKE_dstebr_work);
}

extern "C" int LAPACKE_sstebr(int n, float *d, float *e) {
    return lapacke_stebr<float>(n, d, e, LAPACKE_sstebr_work);
}

// ------------------------------------------------------------ eigenvectors
namespace {

// Workspace of the vector path: the checkpointing layout of the values
// solve, then two buffers for the eigenvector blocks of consecutive levels
// (node g's block at gstart * mmax of its level, n x ceil(n/2) doubles at
// most below the top), the root columns of M of one level and their
// products (n x Kmax each), the GEMM pointer tables, the row signs and the
// per-level Kmax.
struct VecLayout {
    size_t ckpt, qa, qb, mm, sgn, kmax, rows, cnt, total;
};

VecLayout vec_layout(const HostForest &hf, long long n) {
    VecLayout v{};
    v.ckpt = align_up(make_layout(hf, true).bytes);
    const size_t half = (size_t)n * (size_t)((n + 1) / 2) * sizeof(double);
    v.qa = align_up(half);
    v.qb = align_up(half);
    v.mm = align_up((size_t)n * (size_t)n * sizeof(double));
    v.sgn = align_up(sizeof(double) * (size_t)n);
    v.kmax = align_up(sizeof(int) * (size_t)(hf.max_levels + 1));
    v.rows = align_up(sizeof(int) * (size_t)n);
    v.cnt = align_up(sizeof(int) * 2 * (size_t)(hf.nn0 + 1));
    v.total = v.ckpt + v.qa + v.qb + v.mm + v.sgn + v.kmax + v.rows + v.cnt;
    return v;
}

} // namespace

extern "C" brdc_status brdc_dstebr_vectors_workspace_size(int64_t n, size_t *bytes) {
    if (bytes == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    if (n <= 0 || n > kMaxVectorOrder) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    const long long off[2] = {0, (long long)n};
    HostForest hf;
    if (!build_forest(1, off, &hf)) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    *bytes = vec_layout(hf, n).total;
    return BRDC_STATUS_SUCCESS;
}

extern "C" brdc_status brdc_dstebr_vectors(brdc_handle h, int64_t n, const double *d_D,
                                           const double *d_E, double *d_W, double *d_Z,
                                           int64_t ldz, void *workspace, size_t workspace_size) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (d_D == nullptr || d_W == nullptr || d_Z == nullptr || (n > 1 && d_E == nullptr)) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    if (n <= 0 || n > kMaxVectorOrder || ldz < n) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    const long long off[2] = {0, (long long)n};
    HostForest hf;
    if (!build_forest(1, off, &hf)) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    const VecLayout V = vec_layout(hf, n);
    if (workspace == nullptr || workspace_size < V.total) {
        return BRDC_STATUS_INVALID_WORKSPACE;
    }
    cudaStream_t s = h->stream;
    const Layout L = make_layout(hf, true);
    const Ws w = carve(workspace, hf, true);
    Forest F{};
    F.B = 1;
    F.max_levels = hf.max_levels;
    F.n0 = n;
    F.L0 = hf.max_levels;
    // values solve with every merge recorded (and the leaves' eigenvectors)
    const brdc_status st = run_forest(h, hf, L, F, w, d_D, d_E, d_W);
    if (st != BRDC_STATUS_SUCCESS) {
        return st;
    }
    char *base = static_cast<char *>(workspace) + V.ckpt;
    double *qa = reinterpret_cast<double *>(base);
    double *qb = reinterpret_cast<double *>(base + V.qa);
    double *M = reinterpret_cast<double *>(base + V.qa + V.qb);
    double *sgn = reinterpret_cast<double *>(base + V.qa + V.qb + V.mm);
    int *dkmax = reinterpret_cast<int *>(base + V.qa + V.qb + V.mm + V.sgn);
    int *vrows = reinterpret_cast<int *>(base + V.qa + V.qb + V.mm + V.sgn + V.kmax);
    int *vcnt = reinterpret_cast<int *>(base + V.qa + V.qb + V.mm + V.sgn + V.kmax + V.rows);
    k_vec_signs<<<1, 1024, 0, s>>>(d_E, n, sgn);
    BRDC_CUDA(h, "brdc.vectors.signs", cudaGetLastError());
    const int Lv = hf.max_levels;
    long long eg = (n + 7) / 8; // one warp per slot, 8 warps a block
    eg = std::max<long long>(1, std::min<long long>(eg, (long long)h->sm_count * 16));
    long long zg = (n * n + 255) / 256;
    zg = std::max<long long>(1, std::min<long long>(zg, (long long)h->sm_count * 16));
    if (Lv == 0) {
        // one leaf: its eigenvector matrix (ld 16) is the answer
        k_vec_out<<<(unsigned)zg, 256, 0, s>>>(w.leafv, 16, n, sgn, d_Z, ldz);
        BRDC_CUDA(h, "brdc.vectors.leaf", cudaGetLastError());
        return BRDC_STATUS_SUCCESS;
    }
    // the largest K of every level sizes its products (the one read back);
    // inside a graph capture nothing can be read, and every level takes
    // its largest node's order instead (the same result, more flops)
    std::vector<int> kmax(Lv, 0);
    cudaStreamCaptureStatus capst = cudaStreamCaptureStatusNone;
    BRDC_CUDA(h, "brdc.vectors.capture", cudaStreamIsCapturing(s, &capst));
    if (capst != cudaStreamCaptureStatusNone) {
        for (int k = 0; k < Lv; ++k) {
            kmax[k] = hf.level_mmax[k];
        }
    } else {
        BRDC_CUDA(h, "brdc.vectors.kmax_zero", cudaMemsetAsync(dkmax, 0, sizeof(int) * Lv, s));
        for (int k = 0; k < Lv; ++k) {
            Ws wl = w;
            level_view(hf, L, w, k, &wl);
            k_vec_kmax<<<1, 256, 0, s>>>(wl.nK, hf.level_nodes[k], dkmax + k);
        }
        BRDC_CUDA(h, "brdc.vectors.kmax", cudaGetLastError());
        BRDC_CUDA(h, "brdc.vectors.kmax_read",
                  cudaMemcpyAsync(kmax.data(), dkmax, sizeof(int) * Lv, cudaMemcpyDeviceToHost, s));
        BRDC_CUDA(h, "brdc.vectors.kmax_sync", cudaStreamSynchronize(s));
        // a failed values solve (its status word set) leaves the counts
        // unwritten: keep the products inside their buffers whatever was read
        for (int k = 0; k < Lv; ++k) {
            kmax[k] = std::min(std::max(kmax[k], 0), (int)hf.level_mmax[k]);
        }
    }
    double *qprev = nullptr, *qcur = qa;
    long long prev_mmax = 16;
    for (int k = 0; k < Lv; ++k) {
        Ws wl = w;
        level_view(hf, L, w, k, &wl);
        const bool top = (k == Lv - 1);
        const long long mmax = hf.level_mmax[k];
        const int Km = kmax[k];
        VArgs va{};
        va.F = F;
        va.w = wl;
        va.M = M;
        va.mstride = std::max(Km, 1);
        va.k = k;
        va.nodes = hf.level_nodes[k];
        va.child = (k == 0) ? wl.leafv : qprev;
        va.leafchild = (k == 0) ? 1 : 0;
        va.child_stride = prev_mmax;
        va.out = top ? d_Z : qcur;
        va.out_stride = mmax;
        va.top = top ? 1 : 0;
        va.ldout = ldz;
        va.sgn = sgn;
        va.rows = vrows;
        va.cnt = vcnt;
        if (top) {
            k_vec_lowner<<<(unsigned)std::max<long long>(1, std::min<long long>((n + 7) / 8, h->sm_count * 8)),
                           256, 0, s>>>(va);
            BRDC_CUDA(h, "brdc.vectors.lowner", cudaGetLastError());
        }
        // M needs no clearing: k_vec_build writes every row of a root
        // column that k_vec_gemm reads (the poles and the members rotated
        // into them, its listed rows), and nothing else of M is read
        // root columns of M; the deflated eigenvectors straight to the blocks
        k_vec_build<<<(unsigned)eg, 256, 0, s>>>(va, n);
        BRDC_CUDA(h, "brdc.vectors.build", cudaGetLastError());
        if (Km == 0) {
            qprev = qcur;
            qcur = (qcur == qa) ? qb : qa;
            prev_mmax = mmax;
            continue;
        }
        // the roots: blockdiag(Q_left, Q_right) * M[:, :K] per node over the
        // surviving rows of M, each column written to its place (k_vec_gemm,
        // FP64 tensor cores)
        k_vec_rows<256><<<(unsigned)hf.level_nodes[k], 256, 0, s>>>(va);
        BRDC_CUDA(h, "brdc.vectors.rows", cudaGetLastError());
        {
            const long long half_rows = (mmax + 1) / 2;
            const dim3 grid((unsigned)((half_rows + kVgBM - 1) / kVgBM),
                            (unsigned)((Km + kVgBN - 1) / kVgBN),
                            (unsigned)(2 * hf.level_nodes[k]));
            k_vec_gemm<<<grid, kVgThreads, 0, s>>>(va);
            BRDC_CUDA(h, "brdc.vectors.gemm", cudaGetLastError());
        }
        qprev = qcur;
        qcur = (qcur == qa) ? qb : qa;
        prev_mmax = mmax;
    }
    return BRDC_STATUS_SUCCESS;
}

// ---------------------------------------------- allocation-free entry point
// Some callers cannot allocate device memory when they need a solve: code
// that runs inside a host callback or a stream-ordered section where
// cudaMalloc/cudaFree would synchronise or are not permitted, plug-ins
// whose host application owns and budgets every device allocation, and
// latency-critical paths that must not risk an allocation failure in the
// middle of their work.  brdc_dstebr_noalloc serves them: it takes only the
// inputs and the output, and its scratch is the statically sized device
// array below, which exists on every GPU the library is loaded on, from
// load until process exit.  Its size bounds the order of one solve.
namespace {
constexpr long long kNoAllocMaxN = 16384;
constexpr size_t kNoAllocBytes = 6291456; // 6 MiB: the workspace of n = 16384 plus headroom
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mutex;
constexpr int kNoAllocMaxDevices = 128;
void *g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device.  The symbol
// name stands for a host-side shadow in host code, so the address must be
// asked for once per device, with that device current.
cudaError_t noalloc_address(int device, void **out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_addr[device] == nullptr) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            return e;
        }
        g_noalloc_addr[device] = p;
    }
    *out = g_noalloc_addr[device];
    return cudaSuccess;
}

// The address looked up by an earlier brdc_dstebr_noalloc call on `device`
// (nullptr when there was none).
cudaError_t noalloc_cached_address(int device, void **out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    *out = (device >= 0 && device < kNoAllocMaxDevices) ? g_noalloc_addr[device] : nullptr;
    return cudaSuccess;
}
} // namespace

extern "C" brdc_status brdc_dstebr_noalloc_get_info(brdc_handle h, int *info) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (info == nullptr) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    void *scratch = nullptr;
    noalloc_cached_address(h->device, &scratch);
    if (scratch == nullptr) {
        set_error(h, 0, BRDC_ERROR_SRC_NONE,
                  "brdc.noalloc: no allocation-free solve on this device yet");
        return BRDC_STATUS_INVALID_VALUE;
    }
    return brdc_get_info(h, scratch, info);
}

extern "C" brdc_status brdc_dstebr_noalloc(brdc_handle h, int64_t n,
                                           const double *d_D, const double *d_E,
                                           double *d_W) {
    if (h == nullptr) {
        return BRDC_STATUS_INVALID_HANDLE;
    }
    if (d_D == nullptr || d_W == nullptr || (n > 1 && d_E == nullptr)) {
        return BRDC_STATUS_INVALID_POINTER;
    }
    if (n <= 0) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    if (n > kNoAllocMaxN) {
        set_error(h, 0, BRDC_ERROR_SRC_NONE,
                  "brdc.noalloc: n exceeds the static scratch limit of 16384");
        return BRDC_STATUS_INVALID_VALUE;
    }
    const long long off[2] = {0, (long long)n};
    HostForest hf;
    if (!build_forest(1, off, &hf)) {
        return BRDC_STATUS_INVALID_VALUE;
    }
    const Layout L = make_layout(hf);
    if (L.bytes > kNoAllocBytes) {
        set_error(h, 0, BRDC_ERROR_SRC_NONE,
                  "brdc.noalloc: workspace exceeds the static scratch");
        return BRDC_STATUS_INVALID_VALUE;
    }
    int device = 0;
    BRDC_CUDA(h, "brdc.noalloc.get_device", cudaGetDevice(&device));
    if (device < 0 || device >= kNoAllocMaxDevices || device != h->device) {
        set_error(h, device, BRDC_ERROR_SRC_NONE,
                  "brdc.noalloc: current device differs from the handle's");
        return BRDC_STATUS_INVALID_VALUE;
    }
    void *scratch = nullptr;
    BRDC_CUDA(h, "brdc.noalloc.symbol_address", noalloc_address(device, &scratch));
    // Every array the solve reads is written earlier in the same solve and
    // k_init clears the header counters, so the contents left by a previous
    // call need no clearing here.
    const Ws w = carve(scratch, hf, false);
    Forest F{};
    F.B = 1;
    F.max_levels = hf.max_levels;
    F.n0 = n;
    F.L0 = hf.max_levels;
    return run_forest(h, hf, L, F, w, d_D, d_E, d_W);
}
