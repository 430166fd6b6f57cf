// dyg_internal.cuh -- device data layout, Philox stream and shared helpers of
// the B200 dyGRASS update path.
//
// HBM layout of one graph (a dynamic CSR with per-row slack):
//   desc[v]   uint2 {offset, degree}: one 8-byte load gives a walker both the
//             row start and its live length.
//   cap[v]    u32 row capacity (slots reserved at `offset`), touched only by
//             commits and compaction, never by walkers.
//   slots[i]  uint2 {column, bits of 1/weight}: the neighbour id and the
//             resistance a walker adds arrive in one 8-byte load (the
//             reference stores them degree floats apart through a pointer
//             table, gpu_graph.cuh:205-235).  1/w is the correctly rounded
//             float reciprocal, so R += 1/w is bit-identical to dividing on
//             every move.
//   wts[i]    f32 weight of slot i (same offsets as slots); read by exports,
//             recovered edges and the weight-proportional mode, never by the
//             uniform walk.
//   top       arena bump pointer; rows that outgrow their capacity move to
//             [top, top + new_cap) and leave a hole reclaimed by compaction.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <string>
#include <vector>

#include "../../include/dyg.h"

namespace dyg {

constexpr uint32_t kFull = 0xFFFFFFFFu;
constexpr uint32_t kDomainIncr = 0u;   // incremental walks
constexpr uint32_t kDomainDecr = 1u;   // decremental walks
constexpr uint32_t kDomainHeur = 2u;   // 2-step fallback walks

// Device error bits (sticky per workspace until read).
constexpr uint32_t kErrVertex = 1u;    // vertex id >= n in a batch
constexpr uint32_t kErrPath = 2u;      // winner re-walk disagreed with its key
constexpr uint32_t kErrArena = 4u;     // arena overflow in a commit
constexpr uint32_t kErrWeight = 8u;    // weight not finite and > 0 in a batch
constexpr uint32_t kErrScan = 16u;     // a scan tile gave up waiting for its predecessor

struct DevGraph {
    uint2 *desc;
    uint32_t *cap;
    uint2 *slots;
    float *wts;
    unsigned long long *top;   // device scalar
    uint64_t arena_cap;        // slots
    uint32_t n;
};

// ------------------------------------------------------------------ Philox
// Philox4x32-10 (Salmon et al., SC'11).  Counter = {draw block, walker,
// update id low, update id high | domain << 24}, key = seed.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ uint32_t pick4(uint4 v, uint32_t i) {
    return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

__host__ __device__ __forceinline__ uint32_t ctr3_of(uint64_t uid, uint32_t domain) {
    return ((uint32_t)(uid >> 32) & 0x00FFFFFFu) | (domain << 24);
}

// Winner key: max conductance 1/R, then lowest walker id; the low bits carry
// the winner's step count.  0 means no walker reached the target.
__device__ __forceinline__ unsigned long long pack_key(float cond, uint32_t walker,
                                                       uint32_t found) {
    return ((unsigned long long)__float_as_uint(cond) << 32) |
           ((unsigned long long)(1023u - walker) << 22) |
           (unsigned long long)(found & 0x3FFFFFu);
}
__host__ __device__ __forceinline__ uint32_t key_walker(unsigned long long k) {
    return 1023u - (uint32_t)((k >> 22) & 0x3FFu);
}
__host__ __device__ __forceinline__ int32_t key_found(unsigned long long k) {
    return k ? (int32_t)(k & 0x3FFFFFu) : -1;
}

// Fixed-point weight of the weight-proportional mode (exact w * 2^32,
// truncated) so that prefix sums are associative and match the host.
__device__ __forceinline__ unsigned long long wq(float w) {
    const double v = (double)w * 4294967296.0;
    if (!(v > 0.0)) return 0ull;
    if (v >= 18446744073709551615.0) return 0xFFFFFFFFFFFFFFFFull;
    return (unsigned long long)v;
}
__device__ __forceinline__ unsigned long long mul_hi32(uint32_t r, unsigned long long total) {
    // floor(r * total / 2^32) for a 96-bit product
    const unsigned long long lo = (unsigned long long)r * (total & 0xFFFFFFFFull);
    const unsigned long long hi = (unsigned long long)r * (total >> 32);
    return hi + (lo >> 32);
}

// ------------------------------------------------------------- long rows
// Rows longer than kBigRow are scanned, moved and edited by a whole block
// (kBigThreads threads) instead of one thread or one small lane group: on
// power-law graphs a hub row holds tens of thousands of slots, and a serial
// scan of it would bound the whole launch.
constexpr uint32_t kBigRow = 256;
constexpr uint32_t kBigThreads = 256;

// First j < deg with slots[off + j].x == y, or ~0u.  Every thread of the block
// calls it; s_best is one shared word.  Tiles of kFindUnroll * blockDim.x
// slots whose loads are all issued before any compare, so a hub row costs a
// few dependent round trips instead of one per 4 * blockDim.x slots, and a
// match ends the scan at the end of its tile.
constexpr uint32_t kFindUnroll = 16;
__device__ __forceinline__ uint32_t block_find(const uint2 *slots, uint32_t off, uint32_t deg,
                                               uint32_t y, uint32_t *s_best) {
    const uint32_t *cols = reinterpret_cast<const uint32_t *>(slots + off);
    for (uint32_t base = 0; base < deg; base += kFindUnroll * blockDim.x) {
        if (threadIdx.x == 0) *s_best = ~0u;
        __syncthreads();
        uint32_t v[kFindUnroll];
#pragma unroll
        for (uint32_t u = 0; u < kFindUnroll; ++u) {
            const uint32_t j = base + u * blockDim.x + threadIdx.x;
            v[u] = j < deg ? cols[2u * j] : ~0u;   // vertex ids are never ~0u
        }
#pragma unroll
        for (uint32_t u = 0; u < kFindUnroll; ++u)
            if (v[u] == y) {   // this thread's first match is its smallest j
                atomicMin(s_best, base + u * blockDim.x + threadIdx.x);
                break;
            }
        __syncthreads();
        const uint32_t b = *s_best;
        __syncthreads();   // every thread has read it before the next reset
        if (b != ~0u) return b;
    }
    return ~0u;
}

// ------------------------------------------------------------- workspace
// Device scratch owned by a graph handle, grown on demand.
struct Buf {
    void *p = nullptr;
    size_t bytes = 0;
};

struct Workspace {
    Buf keys;                                 // u64 per edge
    Buf flags, pos;                           // u32 per edge
    Buf f_src, f_dst, f_idx;                  // walk list (filtered deletions / new insertions)
    Buf f_uid;                                // u64 per walk-list entry
    Buf f_w;                                  // f32 per walk-list entry (insertions)
    Buf found;                                // u8 per half-edge
    Buf hx, hy, hw;                           // half-edge lists (u32/f32)
    Buf path_v, path_s;                       // winner paths: vertices, taken slots
    Buf path_len;                             // i32 per filtered edge
    Buf cand_x, cand_y, cand_w;               // recovery candidates
    Buf keep;                                 // u32 per candidate
    Buf htab_k, htab_v;                       // dedup hash table
    Buf nop;                                  // u32 no-path filtered indices
    Buf cub_tmp;
    Buf scan_status;                          // u64 per tile of the single-pass scan
    unsigned long long scan_tickets = 0;      // tile tickets handed out so far (S_SCAN)
    uint32_t scan_epoch = 0;                  // tags this workspace's scan statuses per call
    Buf s_src, s_dst, s_w, s_o1, s_o2, s_o3;  // whole-stream staging
    Buf rx2, ry2;                             // recovered edges of a whole stream
    Buf rk2;
    Buf rank, lneed, dtmp;                    // row operations: per-entry rank / need / run
    Buf rowcnt, rowtmp;                       // row operations: per-row counter / run base
    Buf tmask;                                // dedup table size (device)
    Buf del_hx, del_hy;                       // deletion half-edges
    Buf st_key, st_val;                       // stream file: (min, max) keys and indices, sorted
    Buf st_pos;                               // stream file: uint4 slot positions in G and H
    Buf st_wapp;                              // stream file: G weight of each new edge
    Buf big;                                  // uint4 per long-row item (block-cooperative pass)
    Buf s_uid;                                // staged per-edge update ids
    Buf scalars;                              // u64 scalars (see Scalar)
    Buf counts;                               // u32 counts (see Count)
    unsigned long long *host_scalars = nullptr;   // pinned mirror
    uint32_t *host_counts = nullptr;              // pinned mirror
};

// Indices into Workspace::scalars (u64, device) and Workspace::counts (u32).
enum Scalar : int {
    S_NEED = 0,       // arena slots a pending append needs (row moves)
    S_CURSOR = 1,     // arena cursor of the moves of that append (follows S_NEED)
    S_OPRAN = 2,      // set when an append took its row ranks
    S_NBIG = 3,       // entries on the long-row list of the current row operation
    S_TMPCUR = 4,     // scratch cursor of a delete (follows S_NBIG)
    S_ERR = 5,        // device error bits (kErr*)
    S_MOVES = 6,      // walker moves (accumulating)
    S_WALKS = 7,      // walks finished (accumulating)
    S_TOP = 8,        // arena bump pointer of the owning graph
    S_WORK = 9,       // work-chunk counter of the persistent walk kernel
    S_HALT = 10,      // halt code of a stream this handle drives (0 = running)
    S_RECCNT = 11,    // recovered edges recorded so far in a decremental stream
    S_RECCAP = 12,    // capacity of the record buffers (follows S_RECCNT)
    S_LONG = 13,      // set by an append that made a row longer than kBigRow
    S_SCAN = 14,      // tile tickets of the single-pass scan (accumulating)
    S_BLOCKS = 15,    // blocks of an append's sizing pass that finished (the last resets it)
    S_NSCALARS = 16
};
enum Count : int {
    C_FILTERED = 0,   // decremental: edges to walk
    C_CANDS = 1,      // recovery candidates
    C_KEPT = 2,       // half-edges of the kept recovery candidates
    C_NOPATH = 3,     // decremental: edges without a path
    C_ACCEPTED = 4,   // incremental: accepted edges
    C_CANDS2 = 5,     // fallback candidates
    C_RANGE = 6,      // walk-list entries of the current range
    C_WALKLIST = 7,   // stream file: new insertions to walk
    C_GHALF = 8,      // stream file: half-edges of the new insertions (G append)
    C_CANDS_ALL = 9,  // recovery candidates: path, then fallback
    C_HHALF = 10,     // incremental: half-edges of the accepted edges (H append)
    C_NCOUNTS = 12
};

// Halt codes: (batch + 1) << 8 | kind << 4 | phase.
constexpr unsigned long long kHaltArena = 1;    // an arena reservation did not fit
constexpr unsigned long long kHaltRecords = 2;  // the recovered-edge buffers are full
constexpr unsigned long long kHaltInvalid = 3;  // a device-resident batch failed its input check
__host__ __device__ __forceinline__ unsigned long long halt_code(uint32_t batch, uint32_t kind,
                                                                 uint32_t phase) {
    return ((unsigned long long)(batch + 1) << 8) | (kind << 4) | phase;
}

struct AppendList {
    const uint32_t *hx, *hy;
    const float *hw;
    const uint32_t *m_dev;   // device length, or null
    uint32_t m_host;         // host length or upper bound
};

}  // namespace dyg

struct dyg_graph {
    int device = 0;
    dyg::DevGraph g{};
    uint32_t slack = 2;
    double headroom = 0.5;
    dyg::Workspace ws;
    uint64_t moves_total = 0, walks_total = 0;
    // Recovered edges recorded by the last decremental call on this handle
    // (as G); they stay in ws.rx2 / ry2 / rk2 until the next such call.
    uint64_t last_rec = 0;
    // The graph has (or may have) a row longer than kBigRow: row operations
    // then send such rows to the block-cooperative kernels.  Without it every
    // row takes the one-thread path (same results, no extra launches).
    bool long_rows = false;
};

namespace dyg {

void set_error(const std::string &msg);
dyg_status cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define DYG_CUDA(call)                                                          \
    do {                                                                        \
        cudaError_t _e = (call);                                                \
        if (_e != cudaSuccess) return ::dyg::cuda_fail(_e, #call, __FILE__, __LINE__); \
    } while (0)

#define DYG_TRY(call)                      \
    do {                                   \
        dyg_status _s = (call);            \
        if (_s != DYG_OK) return _s;       \
    } while (0)

dyg_status ensure(Buf &b, size_t bytes);
// Where a caller's pointer lives as seen from `device`: host memory (pageable
// or pinned), device memory this device's kernels may read (its own, or
// managed), or device memory of another GPU, which a kernel on `device`
// must not be given.
enum PtrPlace : int { kOnHost = 0, kOnDevice = 1, kOnOtherDevice = 2 };
PtrPlace ptr_place(const void *p, int device);
// DYG_EINVAL (with the argument's name in the message) if any non-null
// pointer of `ptrs` is device memory of another GPU than `device`.
dyg_status check_same_device(int device, const void *const *ptrs, const char *const *names,
                             int count);
template <typename T>
inline T *ptr(const Buf &b) { return static_cast<T *>(b.p); }

int num_sms();
// Counts launches of this library's own kernels (not cub's).
void count_launch();

// --- walk.cu
struct WalkJob {
    const unsigned long long *halt;  // kernels return at once when *halt != 0 (may be null)
    const uint32_t *src, *dst;
    const float *w;              // incremental: per-edge weight; else null
    const unsigned long long *uid;   // per-edge update id, or null -> uid0 + e
    unsigned long long uid0;
    const uint32_t *n_dev;       // device edge count, or null -> n_host
    uint32_t n_host;
    uint32_t domain;
};
dyg_status launch_walk(dyg_graph *G, const WalkJob &job, const dyg_walk_params &p, bool incremental,
                       unsigned long long *keys, cudaStream_t st);
dyg_status launch_walk_scalars(const DevGraph &g, const WalkJob &job, const dyg_walk_params &p,
                               bool incremental, unsigned long long *keys,
                               unsigned long long *scalars, cudaStream_t st);
dyg_status launch_winner_paths(dyg_graph *G, const WalkJob &job, const dyg_walk_params &p,
                               const unsigned long long *keys, uint32_t n_max, uint32_t path_stride,
                               uint32_t *path_v, uint32_t *path_s, int32_t *path_len, cudaStream_t st);
// Writes its candidates at cx/cy/cw + *base_dev.
dyg_status launch_fallback_walks(dyg_graph *G, const unsigned long long *halt,
                                 const uint32_t *f_src, const uint32_t *f_dst,
                                 const unsigned long long *f_uid, const uint32_t *nop,
                                 const uint32_t *n_nop_dev, uint32_t n_nop_max,
                                 const dyg_walk_params &p, const uint32_t *base_dev, uint32_t *cx,
                                 uint32_t *cy, float *cw, cudaStream_t st);

// --- capi.cu
// After a run: DYG_OK, or the error the kernels flagged in G's scalars (last
// read by the run), which are cleared.
dyg_status device_errors(dyg_graph *G, cudaStream_t st);
// DYG_OK, or DYG_EINVAL with the message set, for walk parameters.
dyg_status check_walk_params(const dyg_walk_params *p);

// --- pipeline.cu
// Checks a device-resident batch before anything else of the call runs: an
// endpoint >= nv (kErrVertex) or a weight that is not finite and > 0
// (kErrWeight, when w is given) sets the error bits and the halt code
// kHaltInvalid, so every later kernel of the call returns at once and the
// graphs stay exactly as they were.
dyg_status validate_enqueue(unsigned long long *halt, unsigned long long *err,
                            const uint32_t *src, const uint32_t *dst, const float *w, uint32_t n,
                            uint32_t nv, cudaStream_t st);
// After a run halted with kHaltInvalid: clears the halt and the error bits of
// D (the handle whose scalars held them) and returns DYG_EINVAL with the
// failed check as the message.
dyg_status rejected_inputs(dyg_graph *D, cudaStream_t st);
// uids (device, may be null): per-edge update ids instead of uid_base + e.
// `during`, if given, runs on the host once the first pass of batches is
// enqueued and before the call waits for them: host work that overlaps the
// device work.
dyg_status incremental_run(dyg_graph *H, dyg_graph *G, const uint32_t *src, const uint32_t *dst,
                           const float *w, uint32_t n, uint32_t B, uint64_t uid_base,
                           const unsigned long long *uids, const dyg_walk_params &p, int32_t *found, float *cond, uint8_t *acc,
                           cudaStream_t st, bool check_inputs = false,
                           const std::function<void()> *during = nullptr);
dyg_status decremental_run(dyg_graph *G, dyg_graph *H, const uint32_t *src, const uint32_t *dst,
                           uint32_t n, uint32_t B, uint64_t uid_base,
                           const unsigned long long *uids, const dyg_walk_params &p,
                           int32_t *status, float *cond, uint64_t *n_rec, cudaStream_t st,
                           bool check_inputs = false,
                           const std::function<void()> *during = nullptr);

dyg_status decr_delete_enqueue(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                               const uint32_t *dst, uint32_t n, uint64_t uid0,
                               const unsigned long long *uids, bool file_orient,
                               unsigned long long *halt, int32_t *status, float *cond,
                               cudaStream_t st);
// keys_given (device, may be null): the walk list's winner keys, computed
// elsewhere (a sharded batch); the walks are then skipped.
dyg_status decr_walk_enqueue(dyg_graph *G, dyg_graph *H, uint32_t f0, uint32_t nf,
                             const uint32_t *F_dev, const dyg_walk_params &p,
                             unsigned long long *halt, uint32_t batch, uint32_t phase0,
                             int32_t *status, float *cond, cudaStream_t st,
                             const unsigned long long *keys_given = nullptr);
dyg_status incr_commit_enqueue(dyg_graph *H, dyg_graph *G, const uint32_t *src,
                               const uint32_t *dst, const float *w, uint32_t n,
                               const unsigned long long *keys, unsigned long long *halt,
                               uint32_t batch, int32_t *found, float *cond, uint8_t *acc,
                               cudaStream_t st);
// Grows b to `bytes`, keeping its first `used` bytes.
dyg_status grow_keep(Buf &b, size_t bytes, size_t used, cudaStream_t st);

// --- stream.cu
uint32_t stream_default_chunk(uint32_t n_vertices);
dyg_status stream_file_run(dyg_graph *G, dyg_graph *H, uint32_t op, const uint32_t *src,
                           const uint32_t *dst, const float *w, uint32_t n, uint64_t uid0,
                           uint32_t chunk, const dyg_walk_params &p, int32_t *status, float *cond,
                           uint64_t *n_rec, cudaStream_t st, bool check_inputs = false);

// --- graph.cu
dyg_status upload_graph(dyg_graph *G, uint32_t n, const uint64_t *row_ptr, const uint32_t *col,
                        const float *w);
dyg_status append_enqueue(dyg_graph *GA, const AppendList &A, dyg_graph *GB, const AppendList *B,
                          unsigned long long *halt, unsigned long long code, cudaStream_t st);
// Deletes list entries (hx[i], hy[i]) from G in list order (fG[i] = 1 when
// found), then from H the entries G found on both sides of their edge (fH).
dyg_status delete_pair_enqueue(dyg_graph *G, dyg_graph *H, const uint32_t *hx, const uint32_t *hy,
                               uint32_t m, uint8_t *fG, uint8_t *fH, unsigned long long *halt,
                               cudaStream_t st);
// Copies both graphs' scalars and counts to the host with one synchronize.
dyg_status read_scalars2(dyg_graph *A, dyg_graph *B, cudaStream_t st);
// Exclusive scan of in[0, m) into out; with m_dev, of in[0, min(m, *m_dev)).
dyg_status exclusive_scan_u32(Workspace &ws, const uint32_t *in, uint32_t *out, uint32_t m,
                              cudaStream_t st, const uint32_t *m_dev = nullptr);
dyg_status compact_graph(dyg_graph *G, cudaStream_t st);
dyg_status grow_arena(dyg_graph *G, uint64_t min_cap, cudaStream_t st);
dyg_status read_scalars(dyg_graph *G, cudaStream_t st);
// Rows of local graph [v0, v0 + n) of a pool graph: load places them at the
// arena top (compacting, then growing, when they do not fit) with columns
// shifted by v0 and sets the range's descriptors; save copies them back
// (columns local again, row order kept); clear empties the range (its old
// slots become a hole that compaction reclaims).  load and save synchronize.
dyg_status load_range(dyg_graph *G, uint32_t v0, uint32_t n, const uint64_t *row_ptr,
                      const uint32_t *col, const float *w, cudaStream_t st);
dyg_status save_range(dyg_graph *G, uint32_t v0, uint32_t n, std::vector<uint64_t> &row_ptr,
                      std::vector<uint32_t> &col, std::vector<float> &w, cudaStream_t st);
dyg_status clear_range(dyg_graph *G, uint32_t v0, uint32_t n, cudaStream_t st);
// A graph of n vertices with no slots and an arena of arena_slots (a pool).
dyg_status create_empty_graph(uint32_t n, uint64_t arena_slots, int device, uint32_t slack,
                              double headroom, dyg_graph **out);
void destroy_graph(dyg_graph *G);

}  // namespace dyg
