// Paired step kernels for the fast numerics (variant 5): the P and the A
// half-steps of one time step in ONE launch.
//
// The unfused kernels (pml_step_unfused.cuh) run each half-step as its own
// launch over the whole batch; the A launch then re-reads from DRAM the P(t)
// that the P launch has just written and the A(t-1) that it has just read,
// because a half-step of 64 shots streams far more than the L2 holds: about
// 81 bytes move per cell of a reverse step where 56 are compulsory. Here a
// launch hands out work items in a fixed order, by a ticket counter:
//
//   P item (shot, column block, row segment): the P half-step of the block's
//     8 rows (forward: then the sources and the recording of the receivers
//     and ring cells it owns; reverse: both field sets, then the ring
//     overwrite and the adjoint sources), then it counts itself done for
//     its (shot, row segment);
//   A item (shot, column block, row segment): waits until the P items of its
//     row segment and of the two neighbouring ones are done (its stencil
//     reaches 4 rows and 4 columns beyond the block), then the A half-step
//     (reverse: both sets and the imaging condition) with P(t) read from L2.
//
// The order issues `lead` P items first, then alternates P and A items, so an
// A item is issued about `lead` items after the P items it needs: long
// enough that they have usually finished, short enough that what they wrote
// and read is still in L2 when the A item reads it. Every item an A item
// waits for holds an earlier ticket (lead >= 2 column blocks), and a CTA takes
// its ticket only once it runs, so each awaited item is running or done:
// the waits always end. They are bounded all the same (a timed-out wait sets
// the device error flag; the host reports it).
//
// With many shots, one ticket counter is the one address every CTA of a
// launch updates; per-shot tickets (OTFWI_PAIRED_PER_SHOT=1) spread the
// updates over one counter per shot: the order is then kept within each
// shot, which is all the waits need, and the hardware's dispatch order
// (shot-major) bounds how many shots are in flight.
//
// Tickets and done counts run on across the launches of one time loop (zeroed
// by the loop's first node): launch t (t = 1 .. T-1) hands out tickets
// [(t-1) N, t N) and a row segment is complete at t * ncb done P items. A
// ticket outside its launch's range -- a launch that began before the one
// before it ended, or one that never ran -- sets the error flag, and so does
// a final count that differs from (T-1) N (k_paired_check after the loop).
//
// Cell arithmetic is that of the unfused kernels (the same device functions):
// results are bit-identical to them.
//
// Measured on one B200 (512^2, 64 shots, 300-step proxy of the gradient):
// 0.47 ms per step at the best lead with one ticket counter, 0.58 with
// per-shot counters, against 0.39 for the unfused kernels, which stay the
// default. The spin on the done counts (an acquire at GPU scope per poll)
// and the 128-register cap shared by P and A items cost more than the L2
// re-reads save.
#pragma once
#include "pml_step_unfused.cuh"
#include "tma.cuh"

namespace otf {

// device error flag bits (Engine::sync reports them)
constexpr int kErrWaitTimeout = 1;    // an mbarrier wait of a TMA kernel timed out
constexpr int kErrDepTimeout = 2;     // a paired A item's wait for its P items timed out
constexpr int kErrTicketRange = 4;    // a paired launch saw tickets outside its range
constexpr int kErrLedger = 8;         // a time loop's unfused launches did not all run

struct PairedParams {
    UnfusedParams U;
    unsigned long long *ticket;  // ticket counter of the time loop: [1], or [n_shots] with per-shot tickets
    unsigned *done;              // [n_shots][nseg] done P items per (shot, row segment)
    int *err;                    // device error flag
    int n_shots;
    int lead;                    // P items issued before the first A item (>= 2 ncb)
    // receivers recorded by each P item (forward): CSR over P items (cb + ncb *
    // sg), padded offset and receiver index
    const int *rec_cta, *rec_cta_off, *rec_cta_id;
};

// Item of ticket k: P item idx (is_p) or A item idx; idx = shot * (ncb *
// nseg) + sg * ncb + cb.
__device__ __forceinline__ void paired_item(unsigned k, unsigned np, unsigned lead, bool &is_p, unsigned &idx)
{
    if (k < lead) {
        is_p = true;
        idx = k;
        return;
    }
    const unsigned m = k - lead, pairs = 2u * (np - lead);
    if (m < pairs) {
        is_p = (m & 1u) == 0u;
        idx = is_p ? lead + (m >> 1) : (m >> 1);
    } else {
        is_p = false;
        idx = (np - lead) + (m - pairs);
    }
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void red_release_add(unsigned *p, unsigned v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bounded wait (one lane) until *p >= target.
__device__ __forceinline__ void wait_geq(const unsigned *p, unsigned target, int *err)
{
    if (ld_acquire(p) >= target)
        return;
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 0; it < kWaitIters; it++) {
        __nanosleep(64);
        if (ld_acquire(p) >= target)
            return;
        if ((it & 63u) == 0 && globaltimer_ns() - t0 > kWaitNs)
            break;
    }
    atomicOr(err, kErrDepTimeout);
}

// Ticket of this CTA within its launch (all lanes), or ~0u after flagging a
// ticket outside [0, n_items). PER_SHOT: one counter per shot (blockIdx.y),
// n_items of that shot.
template <bool PER_SHOT>
__device__ __forceinline__ unsigned paired_ticket(const PairedParams &Q, unsigned n_items)
{
    unsigned long long k = 0;
    if (threadIdx.x == 0)
        k = atomicAdd(Q.ticket + (PER_SHOT ? blockIdx.y : 0), 1ull) - (unsigned long long)(Q.U.p.t - 1) * n_items;
    k = __shfl_sync(0xffffffffu, k, 0);
    if (k >= n_items) {
        if (threadIdx.x == 0)
            atomicOr(Q.err, kErrTicketRange);
        return ~0u;
    }
    return (unsigned)k;
}

// A P item's end: every lane's writes ordered before the done count.
__device__ __forceinline__ void paired_release(const PairedParams &Q, int shot, int sg)
{
    __threadfence();
    __syncwarp();
    if (threadIdx.x == 0)
        red_release_add(Q.done + (int64_t)shot * Q.U.nseg + sg, 1u);
}

// An A item's start: its own and both neighbouring row segments complete.
__device__ __forceinline__ void paired_acquire(const PairedParams &Q, int shot, int sg)
{
    if (threadIdx.x == 0) {
        const unsigned target = (unsigned)Q.U.p.t * (unsigned)Q.U.ncb;
        const unsigned *d = Q.done + (int64_t)shot * Q.U.nseg;
        for (int s = max(0, sg - 1); s <= min(Q.U.nseg - 1, sg + 1); s++)
            wait_geq(d + s, target, Q.err);
    }
    __syncwarp();
}

// The item of this CTA: global tickets order every shot's items (grid (2 *
// n_shots * ncb * nseg)); per-shot tickets order one shot's (grid (2 * ncb *
// nseg, n_shots)).
template <bool PER_SHOT>
__device__ __forceinline__ bool paired_take(const PairedParams &Q, bool &is_p, unsigned &idx)
{
    const unsigned nc = (unsigned)(Q.U.ncb * Q.U.nseg);
    const unsigned np = PER_SHOT ? nc : nc * (unsigned)Q.n_shots;
    const unsigned k = paired_ticket<PER_SHOT>(Q, 2u * np);
    if (k == ~0u)
        return false;
    paired_item(k, np, (unsigned)Q.lead, is_p, idx);
    if (PER_SHOT)
        idx += blockIdx.y * nc;
    return true;
}

// Forward step.
template <int MINB, bool PER_SHOT>
__global__ void __launch_bounds__(kUThreads, MINB) k_paired_fwd(const __grid_constant__ PairedParams Q)
{
    pdl_enter();
    const UnfusedParams &U = Q.U;
    const StepParams &p = U.p;
    const unsigned nc = (unsigned)(U.ncb * U.nseg);
    bool is_p;
    unsigned idx;
    if (!paired_take<PER_SHOT>(Q, is_p, idx))
        return;
    const int shot = (int)(idx / nc), w = (int)(idx % nc), sg = w / U.ncb, cb = w % U.ncb;
    const int x = cb * kUCols + 4 * (int)threadIdx.x;
    if (is_p) {
        if (x < p.X)
            p_segment<false>(U, p.f0, p.q0, shot, x, sg * kURows);
        __syncwarp();
        cta_inject(p, p.f0, shot, U.src_cta, U.src_off, U.src_ptr, U.src_id, w, true);
        __syncwarp();
        // recording of the cells this item owns, after their sources
        const float *P = p.f0.px_out + p.shot_stride * shot;
        for (int c = Q.rec_cta[w] + (int)threadIdx.x; c < Q.rec_cta[w + 1]; c += kUThreads)
            p.rec[((int64_t)shot * p.n_sen + Q.rec_cta_id[c]) * p.T + p.t] = P[Q.rec_cta_off[c]];
        if (U.record_ring) {
            float *ring = p.ring + ((int64_t)shot * p.T + p.t) * p.n_ring;
            for (int c = U.ring_cta[w] + (int)threadIdx.x; c < U.ring_cta[w + 1]; c += kUThreads)
                ring[U.ring_cta_k[c]] = P[U.ring_cta_off[c]];
        }
        paired_release(Q, shot, sg);
    } else {
        paired_acquire(Q, shot, sg);
        if (x < p.X)
            a_fwd_segment<true>(U, shot, x, sg * kURows);
    }
}

// Reverse step: a P item updates both field sets of its block.
template <int MINB, bool PER_SHOT>
__global__ void __launch_bounds__(kUThreads, MINB) k_paired_rev(const __grid_constant__ PairedParams Q)
{
    pdl_enter();
    const UnfusedParams &U = Q.U;
    const StepParams &p = U.p;
    const unsigned nc = (unsigned)(U.ncb * U.nseg);
    bool is_p;
    unsigned idx;
    if (!paired_take<PER_SHOT>(Q, is_p, idx))
        return;
    const int shot = (int)(idx / nc), w = (int)(idx % nc), sg = w / U.ncb, cb = w % U.ncb;
    const int x = cb * kUCols + 4 * (int)threadIdx.x;
    if (is_p) {
        if (x < p.X) {
            p_segment<true>(U, p.f0, p.q0, shot, x, sg * kURows);
            p_segment<false>(U, p.f1, p.q1, shot, x, sg * kURows);
        }
        __syncwarp();
        // setRec: P_rec(t) = ring(T-1-t) on the ring cells of this item
        const float *ring = p.ring + ((int64_t)shot * p.T + (p.T - 1 - p.t)) * p.n_ring;
        for (int c = U.ring_cta[w] + (int)threadIdx.x; c < U.ring_cta[w + 1]; c += kUThreads)
            p.f0.px_out[p.shot_stride * shot + U.ring_cta_off[c]] = ring[U.ring_cta_k[c]];
        cta_inject(p, p.f1, shot, U.rcv_cta, U.rcv_off, U.rcv_ptr, U.rcv_id, w, false);
        paired_release(Q, shot, sg);
    } else {
        paired_acquire(Q, shot, sg);
        if (x < p.X)
            a_rev_segment<true>(U, shot, x, sg * kURows);
    }
}

// After a loop of unfused launches: as many launches counted as issued, or
// the error flag.
__global__ void k_ledger_check(const unsigned *ledger, unsigned expect, int *err)
{
    if (*ledger != expect)
        atomicOr(err, kErrLedger);
}

// After a loop of paired launches: every ticket handed out exactly once (n
// counters), or the error flag.
__global__ void k_paired_check(const unsigned long long *ticket, int n, unsigned long long expect, int *err)
{
    for (int i = 0; i < n; i++)
        if (ticket[i] != expect)
            atomicOr(err, kErrTicketRange);
}

}  // namespace otf
