// wavefront.cuh -- the photon march split into two kernels that alternate over a resident pool of
// photon slots (the production path of every plan).
//
// The persistent kernel in march.cuh keeps each photon in one lane for its whole life, so a warp
// mixes marching lanes with lanes that run the discrete logic between marches, and the event code
// sets the register budget (116 registers, 16 warps per SM) of the ER-step loop. Here the two are
// separate kernels over a pool of slots whose state lives in global memory:
//
//   wf_march_kernel  -- every slot on the current march list advances up to `chunk` ER steps
//                       (traceTillBlock, scene.cpp:385-425). Only the march state is loaded
//                       (88 bytes, structure-of-arrays, coalesced), so the kernel runs at a small
//                       register count and high occupancy with no event code in its instruction
//                       stream. Slots whose march ended go to the event queue; the rest go
//                       straight to the next march list.
//   wf_event_kernel  -- every queued slot runs its discrete logic (run_events: face normal, Fresnel
//                       BSDF, sensor connection, splat, HG scattering, roulette) until its next
//                       march starts; a slot whose photon ends takes the next photon index. Slots
//                       that march again are appended to the next march list.
//
// The host alternates the two (march list and event queue double-buffered by iteration parity)
// until the march list is empty. Each kernel resets the counters the other one fills next, so no
// extra launch is needed. Per-photon arithmetic is the same code as the persistent kernel
// (march_step, run_events), so every photon's result is identical.
#pragma once
#include <cuda.h>

#include "march.cuh"

namespace smp {

#ifndef SMP_WF_MARCH_MIN_BLOCKS
#define SMP_WF_MARCH_MIN_BLOCKS 6
#endif

// the state march_step reads and writes
struct MarchState {
    float3 mp, md, mg;
    float mn, cur, dist_acc, dlimit, s, mtotf, hh;
    double mtot, cur_d;
    int steps, end, prec, stop;
    const float4 *tab;
    const Inst *inst;          // batched sweep only
};

// the rest of a Lane, stored per slot as one 128-byte record moved with 16-byte accesses
struct __align__(16) EventPart {
    long long idx;
    double total;
    long long spos, send;
    float3 pos, dir;
    float totalDist;
    int depth, nspl, draws;
    unsigned r0, r1, r2, r3, rblk;
    int rhave, ctx, first;
    float large, d2s, rem, sampled;
    int inst;                  // batched sweep: instance index
};
static_assert(sizeof(EventPart) % 16 == 0, "EventPart is moved as float4s");

__device__ __forceinline__ void ev_load(const EventPart *src, EventPart &E) {
    const float4 *s = reinterpret_cast<const float4 *>(src);
    float4 *d = reinterpret_cast<float4 *>(&E);
#pragma unroll
    for (int i = 0; i < int(sizeof(EventPart) / 16); ++i) d[i] = s[i];
}
__device__ __forceinline__ void ev_store(EventPart *dst, const EventPart &E) {
    float4 *d = reinterpret_cast<float4 *>(dst);
    const float4 *s = reinterpret_cast<const float4 *>(&E);
#pragma unroll
    for (int i = 0; i < int(sizeof(EventPart) / 16); ++i) d[i] = s[i];
}

struct WaveParams {
    // march state, structure of arrays
    float4 *ma;        // mp.xyz, mn
    float4 *mb;        // md.xyz, cur
    float4 *mc;        // mg.xyz, dist_acc
    float4 *mdd;       // dlimit, s, mtotf, instance index (bits; batched sweep)
    int4 *mi;          // steps, end, prec, stop
    double *mt;        // mtot (FP64 path-length form only)
    EventPart *ev;
    int *list[2];      // march lists, by iteration parity
    int *queue[2];     // event queues, by iteration parity
    // Lists and queues hold two classes of march (when `split`): sensor marches (the direct march
    // and connections, CTX_DIRECT / CTX_CONNECT) from the front of the array, moves from its back
    // (entry k of class 1 at n_slots - 1 - k). A warp then marches, and afterwards runs the events
    // of, marches of one kind: long marches to the sensor apart from short exponential moves, and
    // splat + scatter apart from vertex + connection logic.
    unsigned *cnt;     // march list of parity p, class c: cnt[2p + c]; event queue: cnt[4 + 2p + c]
    int split;         // 1: two classes; 0 (spline bricks): class 0 only
    int n_slots;
    int chunk;         // ER steps per slot per march launch (grows when few slots are live)
    // Spline bricks (FK_SPLINE; nb == 0 without them): the march lists binned by the brick of
    // kSplineBrick^3 grid cells each slot's march position lies in -- per parity, brick b's list is
    // blist[par][b * n_slots ...] with bcnt[par][b] entries (cnt[par] still counts them all) -- so a
    // block of the march kernel marches one brick's slots with that brick's coefficients staged in
    // shared memory.
    int *blist[2];
    unsigned *bcnt[2];
    int nb, nbx, nby, nbz;
    int bstride;               // capacity of one brick's list (>= n_slots)
    const float4 *bquads;      // the x-tap quads with their y and z rows padded by -1 .. +2 (mirrored):
                               // N0 x (N1 + 3) x (N2 + 3), the fallback copy's source
    int bdim[3];               // N0, N1 + 3, N2 + 3
    CUtensorMap bmap;          // tiled TMA map of bquads as floats {4, N0, N1 + 3, N2 + 3}, box
                               // {4, kSplineBrick, kSplineBrickRows, kSplineBrickRows}
};

__device__ __forceinline__ unsigned *list_cnt(const WaveParams &W, int par) { return W.cnt + 2 * par; }
__device__ __forceinline__ unsigned *queue_cnt(const WaveParams &W, int par) { return W.cnt + 4 + 2 * par; }
// the march class of a lane about to march: 0 sensor march, 1 move
__device__ __forceinline__ bool move_class(const WaveParams &W, int ctx) {
    return W.split && (ctx == CTX_MOVE_FIRST || ctx == CTX_MOVE_VERTEX);
}
// entry i of a two-class list whose class 0 holds n0 entries
__device__ __forceinline__ int two_class_at(const int *arr, unsigned n0, int n_slots, unsigned i) {
    return i < n0 ? arr[i] : arr[n_slots - 1 - int(i - n0)];
}

// the brick (cells kSplineBrick b .. kSplineBrick b + kSplineBrick - 1 per axis) a march position lies
// in, clamped to the grid
__device__ __forceinline__ int spline_brick_of(const FieldParams &F, const WaveParams &W, float3 p) {
    const float t[3] = {(p.x - F.xmin[0]) * F.xres[0], (p.y - F.xmin[1]) * F.xres[1], (p.z - F.xmin[2]) * F.xres[2]};
    const int nbs[3] = {W.nbx, W.nby, W.nbz};
    int b[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float c = fminf(fmaxf(floorf(t[a]), 0.0f), float(F.N[a] - 1));    // NaN -> 0
        b[a] = min(int(c) / kSplineBrick, nbs[a] - 1);
    }
    return (b[2] * W.nby + b[1]) * W.nbx + b[0];
}

// Appends `slot` of every lane in `mask` to the list of its brick (parity par) and counts them in
// the march-list count of parity par: one atomic per warp for the count and one per group of lanes of the same brick. All 32
// lanes call it.
__device__ __forceinline__ void brick_append(const WaveParams &W, int par, unsigned mask, int brick, int slot, int lane) {
    if (mask == 0u) return;
    if (lane == __ffs(mask) - 1) atomicAdd(list_cnt(W, par), unsigned(__popc(mask)));
    if (mask & (1u << lane)) {
        const unsigned same = __match_any_sync(mask, brick);
        const int leader = __ffs(same) - 1;
        unsigned base = 0u;
        if (lane == leader) base = atomicAdd(W.bcnt[par] + brick, unsigned(__popc(same)));
        base = __shfl_sync(same, base, leader);
        W.blist[par][size_t(brick) * size_t(W.bstride) + base + unsigned(__popc(same & ((1u << lane) - 1u)))] = slot;
    }
}

// live march slot number i of parity par, counted across the brick lists in brick order
__device__ __forceinline__ int brick_slot(const WaveParams &W, int par, unsigned i) {
    int b = 0;
    unsigned acc = 0u;
    while (b < W.nb - 1 && acc + W.bcnt[par][b] <= i) acc += W.bcnt[par][b++];
    return W.blist[par][size_t(b) * size_t(W.bstride) + (i - acc)];
}

__device__ __forceinline__ void wf_load_march(const WaveParams &W, const KParams &P, int slot, MarchState &M) {
    const float4 a = W.ma[slot], b = W.mb[slot], c = W.mc[slot], d = W.mdd[slot];
    const int4 e = W.mi[slot];
    M.mp = f3(a.x, a.y, a.z); M.mn = a.w;
    M.md = f3(b.x, b.y, b.z); M.cur = b.w;
    M.mg = f3(c.x, c.y, c.z); M.dist_acc = c.w;
    M.dlimit = d.x; M.s = d.y; M.mtotf = d.z;
    M.steps = e.x; M.end = e.y; M.prec = e.z; M.stop = e.w;
    M.inst = P.n_inst ? P.insts + __float_as_int(d.w) : nullptr;
    M.hh = 0.5f * M.cur;
    M.cur_d = double(M.cur);
    M.mtot = P.fp64 ? W.mt[slot] : 0.0;
}

template <class S>
__device__ __forceinline__ void wf_store_march(const WaveParams &W, const KParams &P, int slot, const S &M) {
    W.ma[slot] = make_float4(M.mp.x, M.mp.y, M.mp.z, M.mn);
    W.mb[slot] = make_float4(M.md.x, M.md.y, M.md.z, M.cur);
    W.mc[slot] = make_float4(M.mg.x, M.mg.y, M.mg.z, M.dist_acc);
    W.mdd[slot] = make_float4(M.dlimit, M.s, M.mtotf, __int_as_float(P.n_inst ? int(M.inst - P.insts) : 0));
    W.mi[slot] = make_int4(M.steps, M.end, M.prec, M.stop);
    if (P.fp64) W.mt[slot] = M.mtot;
}

__device__ __forceinline__ void wf_load_lane(const WaveParams &W, const KParams &P, int slot, Lane &L) {
    MarchState M;
    wf_load_march(W, P, slot, M);
    L.mp = M.mp; L.mn = M.mn; L.md = M.md; L.cur = M.cur; L.mg = M.mg; L.dist_acc = M.dist_acc;
    L.dlimit = M.dlimit; L.s = M.s; L.mtotf = M.mtotf; L.mtot = M.mtot;
    L.steps = M.steps; L.end = M.end; L.prec = M.prec; L.stop = M.stop;
    L.hh = M.hh; L.cur_d = M.cur_d; L.inst = M.inst;
    EventPart E;
    ev_load(W.ev + slot, E);
    L.idx = E.idx; L.total = E.total; L.spos = E.spos; L.send = E.send;
    L.pos = E.pos; L.dir = E.dir; L.totalDist = E.totalDist;
    L.depth = E.depth; L.nspl = E.nspl; L.draws = E.draws;
    L.r0 = E.r0; L.r1 = E.r1; L.r2 = E.r2; L.r3 = E.r3; L.rblk = E.rblk; L.rhave = E.rhave;
    L.ctx = E.ctx; L.first = E.first;
    L.large = E.large; L.d2s = E.d2s; L.rem = E.rem; L.sampled = E.sampled;
}

__device__ __forceinline__ void wf_store_lane(const WaveParams &W, const KParams &P, int slot, const Lane &L) {
    wf_store_march(W, P, slot, L);
    EventPart E;
    E.idx = L.idx; E.total = L.total; E.spos = L.spos; E.send = L.send;
    E.pos = L.pos; E.dir = L.dir; E.totalDist = L.totalDist;
    E.depth = L.depth; E.nspl = L.nspl; E.draws = L.draws;
    E.r0 = L.r0; E.r1 = L.r1; E.r2 = L.r2; E.r3 = L.r3; E.rblk = L.rblk; E.rhave = L.rhave;
    E.ctx = L.ctx; E.first = L.first;
    E.large = L.large; E.d2s = L.d2s; E.rem = L.rem; E.sampled = L.sampled;
    E.inst = P.n_inst ? int(L.inst - P.insts) : 0;
    ev_store(W.ev + slot, E);
}

// Appends `v` of every lane in `mask` to arr[], one atomic per warp. All 32 lanes call it.
__device__ __forceinline__ void warp_append(int *arr, unsigned *cnt, unsigned mask, int v, int lane) {
    if (mask == 0u) return;
    const int leader = __ffs(mask) - 1;
    unsigned base = 0u;
    if (lane == leader) base = atomicAdd(cnt, unsigned(__popc(mask)));
    base = __shfl_sync(kFull, base, leader);
    if (mask & (1u << lane)) arr[base + unsigned(__popc(mask & ((1u << lane) - 1u)))] = v;
}

// Appends `v` of every lane in `mask` to the two-class array arr[] with counts c[0], c[1]: lanes
// with cls1 to class 1 (from the back), the others to class 0. All 32 lanes call it.
__device__ __forceinline__ void warp_append2(int *arr, unsigned *c, int n_slots, unsigned mask, bool cls1, int v,
                                             int lane) {
    const unsigned m1 = __ballot_sync(kFull, cls1) & mask, m0 = mask & ~m1;
    warp_append(arr, c, m0, v, lane);
    if (m1 == 0u) return;
    const int leader = __ffs(m1) - 1;
    unsigned base = 0u;
    if (lane == leader) base = atomicAdd(c + 1, unsigned(__popc(m1)));
    base = __shfl_sync(kFull, base, leader);
    if (m1 & (1u << lane)) arr[n_slots - 1 - int(base + unsigned(__popc(m1 & ((1u << lane) - 1u))))] = v;
}

// March launch `it` (BLOCK threads per block, a choice of the plan's tuner): slots on list[it & 1]
// advance up to `chunk` ER steps each. When fewer slots
// are live than the grid has lanes, the chunk grows in proportion (up to 64x) so the last photons
// are not paced by launch latency. F64: the FP64 path-length form (only its accumulator is
// loaded, carried and stored).
template <int FK, int F64, int BLOCK>
__global__ void __launch_bounds__(BLOCK, (FK == FK_SPLINE ? 4 : SMP_WF_MARCH_MIN_BLOCKS) * 128 / BLOCK)
wf_march_kernel(const __grid_constant__ KParams P, const __grid_constant__ WaveParams W, int it) {
    extern __shared__ __align__(16) float4 smem_tab[];
    const int lane = threadIdx.x & 31, cur = it & 1, nxt = cur ^ 1;
    const unsigned n0 = list_cnt(W, cur)[0], n = n0 + list_cnt(W, cur)[1];
    if (n == 0u) return;
    if (FK <= FK_BESSELN) {
        if (!stage_to_shared(smem_tab, P.field.btab, unsigned(P.field.bnodes) * 16u, P.counters + CNT_STAGE_TIMEOUT)) {
            // timed out (recorded in the counters): copy with plain loads; a late bulk copy
            // writes the same bytes
            for (int i = threadIdx.x; i < P.field.bnodes; i += blockDim.x) smem_tab[i] = P.field.btab[i];
            __syncthreads();
        }
    }
    const unsigned lanes = gridDim.x * blockDim.x;
    const int chunk = W.chunk * int(min(64u, max(1u, lanes / n)));
    const unsigned nwarps = lanes >> 5;
    unsigned done = 0;                               // ER steps this lane executed
    for (unsigned base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; base < n; base += nwarps * 32u) {
        const unsigned i = base + unsigned(lane);
        const bool valid = i < n;
        bool ended = false;
        int slot = 0;
        if (valid) {
            slot = two_class_at(W.list[cur], n0, W.n_slots, i);
            MarchState M;
            const float4 a = W.ma[slot], b = W.mb[slot], c = W.mc[slot], d = W.mdd[slot];
            const int4 e = W.mi[slot];
            M.mp = f3(a.x, a.y, a.z); M.mn = a.w;
            M.md = f3(b.x, b.y, b.z); M.cur = b.w;
            M.mg = f3(c.x, c.y, c.z); M.dist_acc = c.w;
            M.dlimit = d.x; M.s = d.y; M.mtotf = d.z;
            M.steps = e.x; M.end = 0; M.prec = e.z; M.stop = e.w;   // a marching slot has no end code
            M.hh = 0.5f * M.cur;
            M.cur_d = double(M.cur);
            M.mtot = F64 ? W.mt[slot] : 0.0;
            if (FK == FK_BATCH) {
                M.inst = P.insts + __float_as_int(d.w);
                M.tab = M.inst->field.btab;
            } else {
                M.tab = FK == FK_SPLINE ? nullptr : smem_tab;   // no staged brick: global quads
            }
            const int steps0 = M.steps;
            for (int k = 0; k < chunk; k += 2) {
                if (march_step<FK, F64>(M, P) || march_step<FK, F64>(M, P)) { ended = true; break; }
            }
            done += unsigned(M.steps - steps0);
            W.ma[slot] = make_float4(M.mp.x, M.mp.y, M.mp.z, M.mn);
            W.mb[slot] = make_float4(M.md.x, M.md.y, M.md.z, M.cur);
            W.mc[slot] = make_float4(M.mg.x, M.mg.y, M.mg.z, M.dist_acc);
            if (F64) W.mt[slot] = M.mtot;
            else W.mdd[slot] = make_float4(M.dlimit, M.s, M.mtotf, d.w);
            W.mi[slot] = make_int4(M.steps, M.end, M.prec, M.stop);
        }
        const unsigned em = __ballot_sync(kFull, valid && ended);
        const unsigned cm = __ballot_sync(kFull, valid && !ended);
        warp_append2(W.queue[cur], queue_cnt(W, cur), W.n_slots, em, i >= n0, slot, lane);
        warp_append2(W.list[nxt], list_cnt(W, nxt), W.n_slots, cm, i >= n0, slot, lane);
    }
    unsigned long long wd = done;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wd += __shfl_down_sync(kFull, wd, o);
    if (lane == 0 && wd) atomicAdd(P.counters + CNT_MARCH_STEPS, wd);
}

// ---- the spline's march kernel with TMA-staged coefficient bricks ------------------------------
// Dynamic shared memory of the brick march kernel: alignment slack, the 16-byte header, the quads.
static constexpr unsigned kBrickSmemBytes = 256u + 16u * unsigned(kSplineBrickQuads);
static constexpr int kMaxBricks = 1024;

// Stages brick (bx, by, bz) of the padded quads into shared memory with one tiled tensor copy
// (cp.async.bulk.tensor.4d, no multicast; the tensor map covers this GPU's memory only) on a
// bounded mbarrier wait. The block's thread 0 issues the copy; `phase` is the barrier's next
// parity. On a timeout the block waits once more (bounded), records the failure and returns false,
// and the caller copies with plain loads; after a failure it stops using the copy engine (use_tma).
__device__ __forceinline__ bool stage_brick_tma(float4 *dst, const WaveParams &W, int bx, int by, int bz,
                                                unsigned bar, unsigned &phase, bool &use_tma,
                                                unsigned long long *err) {
    if (!use_tma) return false;
    const unsigned bytes = 16u * unsigned(kSplineBrickQuads);
    if (threadIdx.x == 0) {
        // the block's earlier reads of this memory (generic proxy) come before the copy's writes
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
            ::"r"(smem_u32(dst)), "l"(reinterpret_cast<unsigned long long>(&W.bmap)), "r"(0), "r"(kSplineBrick * bx),
              "r"(kSplineBrick * by), "r"(kSplineBrick * bz), "r"(bar)
            : "memory");
    }
    bool ok = mbar_wait_bounded(bar, phase, 1 << 22);
    if (!ok) {
        ok = mbar_wait_bounded(bar, phase, 1 << 22);       // the copy may still land: wait for it once more
        if (threadIdx.x == 0) atomicAdd(err, 1ull);
    }
    ok = __syncthreads_and(ok ? 1 : 0) != 0;
    if (ok) phase ^= 1u;
    else use_tma = false;
    return ok;
}

// The brick with plain loads (the TMA copy's fallback), zero outside the padded grid as the tensor
// copy fills it.
__device__ __forceinline__ void stage_brick_loads(float4 *dst, const WaveParams &W, int bx, int by, int bz) {
    for (int i = threadIdx.x; i < kSplineBrickQuads; i += blockDim.x) {
        const int x = i % kSplineBrick, y = (i / kSplineBrick) % kSplineBrickRows, z = i / (kSplineBrick * kSplineBrickRows);
        const int gx = kSplineBrick * bx + x, gy = kSplineBrick * by + y, gz = kSplineBrick * bz + z;
        float4 q = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (gx < W.bdim[0] && gy < W.bdim[1] && gz < W.bdim[2])
            q = W.bquads[(size_t(gz) * W.bdim[1] + gy) * W.bdim[0] + gx];
        dst[i] = q;
    }
}

// March launch `it` of a spline plan with bricks. The list of parity it & 1 is binned by brick; the
// kernel walks it in groups of BLOCK slots of one brick (grid-stride over the groups of all bricks,
// in brick order), stages each new brick's coefficients with the Tensor Memory Accelerator, and
// marches the group's slots as wf_march_kernel does, their spline evaluations reading the brick in
// shared memory (a point whose taps leave the brick reads the global quads). Slots whose march
// continues are binned by the brick they now lie in.
template <int F64, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 256 / BLOCK)
wf_march_spline_kernel(const __grid_constant__ KParams P, const __grid_constant__ WaveParams W, int it) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned s_pref[kMaxBricks + 1];
    __shared__ __align__(8) unsigned long long s_bar;
    const int lane = threadIdx.x & 31, cur = it & 1, nxt = cur ^ 1;
    const unsigned n = list_cnt(W, cur)[0];                 // one class: no split with bricks
    if (n == 0u) return;
    // the brick: quads 128-byte aligned, the header in the 16 bytes before them
    float4 *quads = reinterpret_cast<float4 *>((reinterpret_cast<uintptr_t>(smem_raw) + 16u + 127u) & ~uintptr_t(127));
    float4 *brick = quads - 1;
    const unsigned bar = smem_u32(&s_bar);
    if (threadIdx.x == 0) {
        unsigned acc = 0u;
        s_pref[0] = 0u;
        for (int b = 0; b < W.nb; ++b) {
            acc += (W.bcnt[cur][b] + unsigned(BLOCK) - 1u) / unsigned(BLOCK);
            s_pref[b + 1] = acc;
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const unsigned groups = s_pref[W.nb];
    const unsigned lanes = gridDim.x * blockDim.x;
    const int chunk = W.chunk * int(min(64u, max(1u, lanes / n)));
    unsigned phase = 0u;
    bool use_tma = true;
    int staged = -1;
    unsigned done = 0;                               // ER steps this lane executed
    for (unsigned g = blockIdx.x; g < groups; g += gridDim.x) {
        // the brick of group g: the last b with s_pref[b] <= g (empty bricks have no groups)
        int lo = 0, hi = W.nb;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_pref[mid] <= g) lo = mid; else hi = mid;
        }
        const int b = lo;
        if (b != staged) {
            __syncthreads();                         // every lane is done with the previous brick
            const int bx = b % W.nbx, by = (b / W.nbx) % W.nby, bz = b / (W.nbx * W.nby);
            if (!stage_brick_tma(quads, W, bx, by, bz, bar, phase, use_tma, P.counters + CNT_STAGE_TIMEOUT)) {
                stage_brick_loads(quads, W, bx, by, bz);
            }
            if (threadIdx.x == 0)
                *reinterpret_cast<int4 *>(brick) = make_int4(kSplineBrick * bx, kSplineBrick * by, kSplineBrick * bz, 1);
            __syncthreads();
            staged = b;
        }
        const unsigned i = (g - s_pref[b]) * unsigned(BLOCK) + threadIdx.x;
        const bool valid = i < W.bcnt[cur][b];
        bool ended = false;
        int slot = 0, key = 0;
        if (valid) {
            slot = W.blist[cur][size_t(b) * size_t(W.bstride) + i];
            MarchState M;
            const float4 a = W.ma[slot], bb = W.mb[slot], c = W.mc[slot], d = W.mdd[slot];
            const int4 e = W.mi[slot];
            M.mp = f3(a.x, a.y, a.z); M.mn = a.w;
            M.md = f3(bb.x, bb.y, bb.z); M.cur = bb.w;
            M.mg = f3(c.x, c.y, c.z); M.dist_acc = c.w;
            M.dlimit = d.x; M.s = d.y; M.mtotf = d.z;
            M.steps = e.x; M.end = 0; M.prec = e.z; M.stop = e.w;   // a marching slot has no end code
            M.hh = 0.5f * M.cur;
            M.cur_d = double(M.cur);
            M.mtot = F64 ? W.mt[slot] : 0.0;
            M.tab = brick;
            M.inst = nullptr;
            const int steps0 = M.steps;
            for (int k = 0; k < chunk; k += 2) {
                if (march_step<FK_SPLINE, F64>(M, P) || march_step<FK_SPLINE, F64>(M, P)) { ended = true; break; }
            }
            done += unsigned(M.steps - steps0);
            W.ma[slot] = make_float4(M.mp.x, M.mp.y, M.mp.z, M.mn);
            W.mb[slot] = make_float4(M.md.x, M.md.y, M.md.z, M.cur);
            W.mc[slot] = make_float4(M.mg.x, M.mg.y, M.mg.z, M.dist_acc);
            if (F64) W.mt[slot] = M.mtot;
            else W.mdd[slot] = make_float4(M.dlimit, M.s, M.mtotf, d.w);
            W.mi[slot] = make_int4(M.steps, M.end, M.prec, M.stop);
            if (!ended) key = spline_brick_of(P.field, W, M.mp);
        }
        const unsigned em = __ballot_sync(kFull, valid && ended);
        const unsigned cm = __ballot_sync(kFull, valid && !ended);
        warp_append(W.queue[cur], queue_cnt(W, cur), em, slot, lane);
        brick_append(W, nxt, cm, key, slot, lane);
    }
    unsigned long long wd = done;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wd += __shfl_down_sync(kFull, wd, o);
    if (lane == 0 && wd) atomicAdd(P.counters + CNT_MARCH_STEPS, wd);
}

// Event launch `it` (or the initial fill when it < 0): queued slots run their discrete logic;
// finished photons are replaced from the global photon counter; slots that start a march are
// appended to the next march list. Also resets the march-list counter just consumed and the event
// queue the next march launch fills.
#ifndef SMP_WF_EVENT_MIN_BLOCKS
#define SMP_WF_EVENT_MIN_BLOCKS 4
#endif
template <int FK>
__global__ void __launch_bounds__(128, SMP_WF_EVENT_MIN_BLOCKS)
wf_event_kernel(const __grid_constant__ KParams P, const __grid_constant__ WaveParams W, int it) {
    const int lane = threadIdx.x & 31;
    const bool init = it < 0;
    const int cur = init ? 1 : (it & 1), nxt = cur ^ 1;
    const unsigned q0 = init ? unsigned(W.n_slots) : queue_cnt(W, cur)[0];
    const unsigned n = init ? q0 : q0 + queue_cnt(W, cur)[1];
    if (!init && blockIdx.x == 0 && threadIdx.x < 2) {
        list_cnt(W, cur)[threadIdx.x] = 0u;     // consumed by march launch `it`
        queue_cnt(W, nxt)[threadIdx.x] = 0u;    // filled by march launch `it + 1`
    }
    if (FK == FK_SPLINE && !init && blockIdx.x == 0)
        for (int b = threadIdx.x; b < W.nb; b += blockDim.x) W.bcnt[cur][b] = 0u;   // the brick lists too
    LaneStats S;
    const unsigned lanes = gridDim.x * blockDim.x, nwarps = lanes >> 5;
    for (unsigned base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; base < n; base += nwarps * 32u) {
        const unsigned i = base + unsigned(lane);
        const bool valid = i < n;
        int st = ST_DONE, slot = 0, key = 0;
        bool cls1 = false;
        if (valid) {
            slot = init ? int(i) : two_class_at(W.queue[cur], q0, W.n_slots, i);
            Lane L;
            if (init) {
                L.end = 0;
                L.idx = 0;
                st = ST_FETCH;
            } else {
                wf_load_lane(W, P, slot, L);
                L.tab = FK == FK_BATCH ? L.inst->field.btab : P.field.btab;
                st = run_events<FK>(L, P, EV_MARCH_END);
                if (st == ST_FETCH) finish_photon_stats<FK>(L, S);
            }
            if (FK != FK_BATCH) L.tab = P.field.btab;         // a batched photon's table is set at its start
            while (st == ST_FETCH) {
                // one atomic per group of lanes that fetch together
                const cg::coalesced_group g = cg::coalesced_threads();
                unsigned long long k = 0;
                if (g.thread_rank() == 0) k = atomicAdd(P.counters + CNT_NEXT_PHOTON, (unsigned long long)g.size());
                k = g.shfl(k, 0) + g.thread_rank();
                if (k < (unsigned long long)P.n_photons) {
                    L.idx = P.first_photon + (long long)k;
                    L.end = 0;
                    st = run_events<FK>(L, P, EV_NEW);
                    if (st == ST_FETCH) finish_photon_stats<FK>(L, S);
                } else {
                    st = ST_DONE;
                }
            }
            if (st == ST_MARCH) {
                wf_store_lane(W, P, slot, L);
                if (FK == FK_SPLINE && W.nb) key = spline_brick_of(P.field, W, L.mp);
                cls1 = move_class(W, L.ctx);
            }
        }
        const unsigned mm = __ballot_sync(kFull, valid && st == ST_MARCH);
        if (FK == FK_SPLINE && W.nb) brick_append(W, nxt, mm, key, slot, lane);
        else warp_append2(W.list[nxt], list_cnt(W, nxt), W.n_slots, mm, cls1, slot, lane);
    }
    flush_stats(S, P, lane);
}

// The tail: once the photon counter is exhausted the live slots drain, and a march launch lasts
// as long as its longest march while slots with short marches wait for the next event launch. When
// the live slots fit in one persistent grid, this kernel loads each into a lane of the persistent
// loop (march and events in one kernel, march.cuh) and runs them to the end. A grid too small for
// the list is a host error, recorded in CNT_LOST.
template <int FK>
__global__ void __launch_bounds__(128, SMP_MIN_BLOCKS)
wf_finish_kernel(const __grid_constant__ KParams P, const __grid_constant__ WaveParams W, int it) {
    extern __shared__ __align__(16) float4 smem_tab[];
    const int lane = threadIdx.x & 31, cur = it & 1;
    const unsigned n0 = list_cnt(W, cur)[0], n = n0 + list_cnt(W, cur)[1];
    const unsigned gid = blockIdx.x * blockDim.x + threadIdx.x, lanes = gridDim.x * blockDim.x;
    if (gid == 0 && n > lanes) atomicAdd(P.counters + CNT_LOST, (unsigned long long)(n - lanes));
    const float4 *tab = P.field.btab;
    if (FK <= FK_BESSELN && P.field.btab != nullptr) {
        if (stage_to_shared(smem_tab, P.field.btab, unsigned(P.field.bnodes) * 16u, P.counters + CNT_STAGE_TIMEOUT))
            tab = smem_tab;
    }
    Lane L;
    L.end = 0;
    L.idx = 0;
    int st = ST_FETCH;
    L.inst = nullptr;
    if (gid < n) {
        wf_load_lane(W, P, (FK == FK_SPLINE && W.nb) ? brick_slot(W, cur, gid) : two_class_at(W.list[cur], n0, W.n_slots, gid), L);
        st = ST_MARCH;
    }
    L.tab = (FK == FK_BATCH && L.inst) ? L.inst->field.btab : tab;
    LaneStats S;
    lane_loop<FK>(L, st, P, S, lane);
    flush_stats(S, P, lane);
}

}  // namespace smp
