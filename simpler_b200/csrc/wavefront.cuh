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
    unsigned *cnt;     // cnt[0..1] march-list lengths, cnt[2..3] event-queue lengths
    int n_slots;
    int chunk;         // ER steps per slot per march launch (grows when few slots are live)
};

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
    const unsigned n = W.cnt[cur];
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
            slot = W.list[cur][i];
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
                M.tab = smem_tab;
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
        warp_append(W.queue[cur], W.cnt + 2 + cur, em, slot, lane);
        warp_append(W.list[nxt], W.cnt + nxt, cm, slot, lane);
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
template <int FK>
__global__ void __launch_bounds__(128, 4)
wf_event_kernel(const __grid_constant__ KParams P, const __grid_constant__ WaveParams W, int it) {
    const int lane = threadIdx.x & 31;
    const bool init = it < 0;
    const int cur = init ? 1 : (it & 1), nxt = cur ^ 1;
    const unsigned n = init ? unsigned(W.n_slots) : W.cnt[2 + cur];
    if (!init && blockIdx.x == 0 && threadIdx.x == 0) {
        W.cnt[cur] = 0u;          // consumed by march launch `it`
        W.cnt[2 + nxt] = 0u;      // filled by march launch `it + 1`
    }
    LaneStats S;
    const unsigned lanes = gridDim.x * blockDim.x, nwarps = lanes >> 5;
    for (unsigned base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; base < n; base += nwarps * 32u) {
        const unsigned i = base + unsigned(lane);
        const bool valid = i < n;
        int st = ST_DONE, slot = 0;
        if (valid) {
            slot = init ? int(i) : W.queue[cur][i];
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
            if (st == ST_MARCH) wf_store_lane(W, P, slot, L);
        }
        const unsigned mm = __ballot_sync(kFull, valid && st == ST_MARCH);
        warp_append(W.list[nxt], W.cnt + nxt, mm, slot, lane);
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
    const unsigned n = W.cnt[cur];
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
        wf_load_lane(W, P, W.list[cur][gid], L);
        st = ST_MARCH;
    }
    L.tab = (FK == FK_BATCH && L.inst) ? L.inst->field.btab : tab;
    LaneStats S;
    lane_loop<FK>(L, st, P, S, lane);
    flush_stats(S, P, lane);
}

}  // namespace smp
