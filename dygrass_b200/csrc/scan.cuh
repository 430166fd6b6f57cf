// scan.cuh -- single-pass exclusive scan of u32 with the producer and the
// consumer of the scanned values fused into the same launch.
//
// Decoupled look-back (Merrill & Garland, "Single-pass Parallel Prefix Scan
// with Decoupled Look-back", 2016): each block takes the next tile in ticket
// order, publishes its tile's sum, then its first warp reads the status words
// of the 32 nearest predecessors at a time, adds their sums back to the
// nearest one holding an inclusive prefix, and publishes the tile's own
// inclusive prefix.  A tile waits only on tiles that took earlier tickets, so
// they are running or done and publish without waiting; the wait is still
// bounded, and a tile that gives up sets kErrScan (the call then fails)
// instead of spinning on.  Status words carry the call's epoch, so no memset
// is needed between calls: (epoch << 34) | (flag << 32) | value, flag 1 =
// tile sum, 2 = inclusive prefix.
//
// The operator supplies the element values and consumes the prefixes:
//   uint32_t load(uint32_t i)                 value of element i (i < m); may
//                                             write per-element side outputs
//   void store(uint32_t i, uint32_t excl, uint32_t v)
//                                             exclusive prefix of element i
//   void last(uint32_t total)                 once, with the sum of [0, m)
// so a flag pass, the scan and the compaction that follows it are one launch.
// With a device count m_dev, the scan covers [0, min(m, *m_dev)); the tiles
// past it leave after their ticket (no tile that stays looks back at them).
// A halted stream (*halt != 0) makes every tile leave after its ticket.
#pragma once

#include "dyg_internal.cuh"

namespace dyg {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;
constexpr uint32_t kScanSpinLimit = 1u << 20;   // about a second of L2 reads

struct ScanCtl {
    unsigned long long *status;   // one word per tile
    unsigned long long *ticket;   // scalars + S_SCAN
    unsigned long long base;      // tickets handed out before this launch
    uint32_t epoch;
    unsigned long long *err;      // scalars + S_ERR
    const unsigned long long *halt;
};

__device__ __forceinline__ unsigned long long scan_word(uint32_t epoch, uint32_t flag, uint32_t v) {
    return ((unsigned long long)(epoch & 0x3FFFFFFFu) << 34) | ((unsigned long long)flag << 32) | v;
}

template <class Op>
__global__ void __launch_bounds__(kScanThreads)
k_scan_op(Op op, uint32_t m, const uint32_t *m_dev, ScanCtl c) {
    __shared__ uint32_t s_tile, s_prefix;
    __shared__ uint32_t s_warp[kScanThreads / 32];
    if (threadIdx.x == 0) {
        const unsigned long long t = atomicAdd(c.ticket, 1ull) - c.base;
        s_tile = t < gridDim.x ? (uint32_t)t : ~0u;
        if (t >= gridDim.x) atomicOr(c.err, (unsigned long long)kErrScan);   // tickets out of step
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile == ~0u) return;
    if (c.halt && *c.halt) return;
    if (m_dev) m = min(m, *m_dev);
    if ((uint64_t)tile * kScanTile >= m) return;
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    const uint64_t i0 = (uint64_t)tile * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int u = 0; u < kScanItems; ++u) {
        v[u] = (i0 + u < m) ? op.load((uint32_t)(i0 + u)) : 0u;
        sum += v[u];
    }
    // block scan of the per-thread sums
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    if (lane == 31u) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < kScanThreads / 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= (uint32_t)o) w += t;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = w;   // inclusive over warps
    }
    __syncthreads();
    const uint32_t before_warp = wid ? s_warp[wid - 1] : 0u;
    const uint32_t tile_sum = s_warp[kScanThreads / 32 - 1];
    if (wid == 0) {
        const uint32_t ep_now = c.epoch & 0x3FFFFFFFu;
        if (tile == 0) {
            if (lane == 0) {
                atomicExch(c.status, scan_word(c.epoch, 2u, tile_sum));
                s_prefix = 0u;
            }
        } else {
            if (lane == 0) atomicExch(c.status + tile, scan_word(c.epoch, 1u, tile_sum));
            volatile unsigned long long *vs = c.status;
            uint32_t excl = 0;
            int64_t j = (int64_t)tile - 1;   // lane l reads predecessor j - l
            uint32_t spins = 0;
            while (true) {
                const int64_t at = j - (int64_t)lane;
                // before tile 0: an inclusive prefix of 0
                const unsigned long long w = at >= 0 ? vs[at] : scan_word(c.epoch, 2u, 0u);
                const uint32_t fl = ((uint32_t)(w >> 34) == ep_now) ? (uint32_t)(w >> 32) & 3u : 0u;
                if (!__all_sync(0xFFFFFFFFu, fl != 0u)) {
                    if (++spins > kScanSpinLimit) {   // warp-uniform
                        if (lane == 0) atomicOr(c.err, (unsigned long long)kErrScan);
                        break;
                    }
                    continue;
                }
                const unsigned inc = __ballot_sync(0xFFFFFFFFu, fl == 2u);
                const uint32_t stop = inc ? (uint32_t)(__ffs(inc) - 1) : 31u;
                excl += __reduce_add_sync(0xFFFFFFFFu, lane <= stop ? (uint32_t)w : 0u);
                if (inc) break;
                j -= 32;
            }
            if (lane == 0) {
                atomicExch(c.status + tile, scan_word(c.epoch, 2u, excl + tile_sum));
                s_prefix = excl;
            }
        }
    }
    __syncthreads();
    uint32_t run = s_prefix + before_warp + incl - sum;
#pragma unroll
    for (int u = 0; u < kScanItems; ++u) {
        if (i0 + u < m) {
            op.store((uint32_t)(i0 + u), run, v[u]);
            if (i0 + u == (uint64_t)m - 1u) op.last(run + v[u]);
        }
        run += v[u];
    }
}

// Enqueues the scan of [0, m) (of [0, min(m, *m_dev)) with a device count).
template <class Op>
dyg_status scan_op(Workspace &ws, const Op &op, uint32_t m, const uint32_t *m_dev,
                   const unsigned long long *halt, cudaStream_t st) {
    if (m == 0) return DYG_OK;
    const uint32_t tiles = (m + kScanTile - 1) / kScanTile;
    if (ws.scan_status.bytes < sizeof(unsigned long long) * tiles) {
        DYG_TRY(ensure(ws.scan_status, sizeof(unsigned long long) * tiles));
        DYG_CUDA(cudaMemsetAsync(ws.scan_status.p, 0, ws.scan_status.bytes, st));
    }
    ws.scan_epoch = ws.scan_epoch + 1u == 0x40000000u ? 1u : ws.scan_epoch + 1u;
    unsigned long long *sc = ptr<unsigned long long>(ws.scalars);
    const ScanCtl c{ptr<unsigned long long>(ws.scan_status), sc + S_SCAN, ws.scan_tickets,
                    ws.scan_epoch, sc + S_ERR, halt};
    k_scan_op<Op><<<tiles, kScanThreads, 0, st>>>(op, m, m_dev, c);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    ws.scan_tickets += tiles;   // every launched tile takes one ticket
    return DYG_OK;
}

}  // namespace dyg
