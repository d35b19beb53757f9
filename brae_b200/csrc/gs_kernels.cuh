// gs_kernels.cuh -- exact Gauss-Seidel (GaussSeidelSmoother::smooth as gaussSeidelSweeps runs it,
// src/OpenFOAM/matrices/smooth_solver_cpp.cu:87-166) on the device, bit for bit.
//
// THE SWEEP IN GATHER FORM. The reference walks cells ascending; cell c's new value is
//     (((b_c - l_f1*psi'[o1]) - l_f2*psi'[o2]) ... - u_g1*psi[n1] - u_g2*psi[n2] ...) / d_c
// where f1, f2, ... are the faces c is the neighbour of, in face order (their owners o < c were
// updated earlier in the sweep and distributed into bPrime in exactly that order), and g1, g2, ...
// the faces c owns (neighbours n > c, still at their old values). As a gather per cell, a cell
// needs only its owners' new values: the sweep is a DAG and a cell's "depth" is its level in it.
//
// SWEEP ORDER. Every vector of a level is stored in "position" order: cells split into P contiguous
// index ranges ("parts", one persistent CTA each), each part's cells by (depth, cell). A part walks
// its positions in order, cut into "chunks" of at most M cells of one depth. Cells of one depth do
// not depend on each other, so a CTA barrier is needed only where the depth changes.
//
// THE CRITICAL PATH. A sweep takes about (DAG depth) x (time per chunk), so everything but the
// row arithmetic is taken off the compute warps:
//   * a PRODUCER warp stages chunk j, S-1 chunks ahead, into one of S shared-memory slots: the
//     chunk's contiguous data (diagonal, b, row descriptors, entry codes, coefficients) by TMA bulk
//     copies, the psi window's old values ahead of the front (TMA), and the values the window does
//     not hold by cp.async gathers; all of it completes on the slot's `full` mbarrier;
//   * a SERVICE warp publishes the part's progress word and polls the upstream parts' words;
//   * the COMPUTE warps (one thread per cell) wait on `full`, compute their rows from shared
//     memory only, and release the slot warp by warp on its `empty` mbarrier.
//
// ENTRY LAYOUT (sliced ELL, per chunk). A chunk's entries are stored in slices of 32 cells (one
// warp): entry q of the cell in lane l of a slice sits at sliceBase + 32*q + l, so a warp reads 32
// consecutive codes and coefficients per entry -- free of shared-memory bank conflicts. A cell's
// row descriptor is width << 24 | (its slice base + lane, relative to the chunk), the width being
// the slice's longest row: every lane of a warp walks the same number of entries, the shorter rows
// padded with entries that read a zero with coefficient zero (acc - 0*0 == acc, so the padding
// leaves the result bit for bit as it is). Codes are 16 bits: bit 15 clear -> window slot
// (position mod W); set -> index into the chunk's gathered values (the last index: the zero).
//
// WHAT THE WINDOW HOLDS. W positions of psi around the front: behind it the part's NEW values
// (written as they are computed), ahead of it the OLD values (filled by TMA as the front advances).
// The schedule (hierarchy.cu) codes an entry as a window read when the value is there for certain
// (gsWindowExtents), else as a gather: old values of neighbours further ahead or in other parts,
// owners further behind (the producer waits until this part has finished their chunk), owners in
// other parts (the producer waits until those parts' progress covers them).
//
// WHY OLD VALUES MAY BE READ EARLY. A neighbour n of a cell c has depth(n) > depth(c), so n is
// rewritten only after c's depth completes: in this part after c's chunk, in another part only after
// that part saw this part's progress pass depth(c), which is published after c's chunk.
//
// BOUNDED WAITS. Every spin has a budget; when it runs out the error word is set and later waits give
// up at once, so a broken schedule ends the kernel with an error instead of hanging the GPU.
#pragma once

#include <cuda_pipeline.h>

#include "b2g_common.cuh"

namespace b2g {
namespace k {

constexpr int kWin = 4096;                     // W: psi window (positions), a power of two
constexpr int kFill = 256;                     // B: window fill block (positions)
constexpr int kStages = 6;                     // S: pipeline slots
constexpr unsigned kGatBit = 0x8000u;          // code bit: gathered value
constexpr int kMaxGat = 0x8000;                // gathered values per chunk, at most
constexpr int kMaxCompute = 448;               // compute threads per CTA, at most (+ 2 warps)
constexpr long long kSpinLimit = 1LL << 24;    // polls before a wait gives up

// Window extents the schedule relies on for a chunk starting at s and ending at e: positions
// [s, s + ahead) hold old values, [e - behind, s) new ones. Fills for chunk j are issued once chunk
// j-S is consumed, so up to S-1 chunks (at most (S-2)*M positions past the oldest one's end) may be
// in flight; they must not overwrite new values a pending chunk still reads:
// ahead + behind + B + (S-2)*M <= W.
inline void gsWindowExtents(int M, int& ahead, int& behind)
{
    const int room = kWin - kFill - (kStages - 2) * M;
    ahead = room / 2;
    behind = room - ahead;
}

// Chunk record, 12 ints (three int4).
struct ChunkRec
{
    int pos0, m, ent0, nEnt;        // positions [pos0, pos0+m); ELL entries [ent0, ent0+nEnt)
    int gat0, nGat, depth, needUp;  // gather list [gat0, gat0+nGat); other-part owners' max depth or -1
    int sameWait, newDepth, pad0, pad1;  // last same-part chunk a gather reads (global index) or -1;
                                         // 1 where the depth changes within the part
};

template <class T>
struct GsArgs
{
    int nParts;
    int maxCells;                  // M: chunk cell capacity (compute threads, a multiple of 32)
    int maxEnt;                    // E: chunk ELL entry capacity (a multiple of 32)
    int maxGat;                    // chunk gather capacity; index maxGat-1 holds the zero
    int ahead;                     // window extent ahead of a chunk's start (positions)
    int nPadded;                   // psi is readable up to here (whole fill blocks)
    const int* __restrict__ partChunkStart;  // [P+1]
    const int* __restrict__ partPosStart;    // [P+1]
    const int4* __restrict__ chunkRec;       // [nChunks][3]
    const int* __restrict__ upStart;         // [P+1]
    const int* __restrict__ upList;
    const int* __restrict__ hasDown;         // [P] 1 if another part reads this part's values
    const unsigned* __restrict__ posEnt;     // [n (+pad)] row descriptor by position
    const unsigned short* __restrict__ entCode;  // [ELL entries]
    const T* __restrict__ entVal;            // [ELL entries]
    const int* __restrict__ gatSrc;          // [gathers] position of each gathered value
    const T* __restrict__ posDiag;           // [n (+pad)]
    const T* __restrict__ b;                 // [n (+pad)] by position
    T* psi;                                  // [n] by position, updated in place (padded)
    unsigned* progress;                      // [P]
    int* err;
    unsigned long long* trace;               // diagnostic, or null: [nChunks][4] clock64 stamps of
                                             // compute thread 0 (start, data ready, computed,
                                             // released), [P][4] {globaltimer, clock64} at the
                                             // part's start and end, [nChunks][2] producer stamps
                                             // (start, copies issued)
};

__device__ __forceinline__ unsigned long long globalTimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned long long clockStamp()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%clock64;" : "=l"(t)::"memory");
    return t;
}

__device__ __forceinline__ unsigned smemAddr(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbarInit(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbarExpectTx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbarArrive(unsigned long long* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(bar)) : "memory");
}
// arrive once this thread's earlier cp.async copies have landed (the arrival is counted in the
// barrier's expected count)
__device__ __forceinline__ void mbarArriveCpAsync(unsigned long long* bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smemAddr(bar)) : "memory");
}
__device__ __forceinline__ bool mbarTryWait(unsigned long long* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smemAddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// 1-D TMA bulk copy global -> shared, completing on `bar`. dst, src 16-byte aligned; bytes % 16 == 0.
__device__ __forceinline__ void tmaLoad(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smemAddr(dst)),
                 "l"(src), "r"(bytes), "r"(smemAddr(bar))
                 : "memory");
}
// Shared-memory accesses by 32-bit address (volatile: they stay ordered against the barrier waits)
__device__ __forceinline__ unsigned ldsU32(unsigned a)
{
    unsigned v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ unsigned ldsU16(unsigned a)
{
    unsigned short v;
    asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ double ldsT(unsigned a, double)
{
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ float ldsT(unsigned a, float)
{
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ void stsT(unsigned a, double v) { asm volatile("st.shared.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory"); }
__device__ __forceinline__ void stsT(unsigned a, float v) { asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory"); }

__device__ __forceinline__ void fenceProxyAsyncShared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// A 16-byte-aligned cover of elements [i0, i0 + cnt) of an array whose base is 16-byte aligned.
struct Cover
{
    const char* src;
    unsigned bytes;
    int lead;  // elements between the cover's start and element i0
};
template <class E>
__host__ __device__ __forceinline__ Cover coverOf(const E* base, long long i0, int cnt)
{
    const long long b0 = i0 * static_cast<long long>(sizeof(E));
    const long long b1 = (i0 + cnt) * static_cast<long long>(sizeof(E));
    const long long a0 = b0 & ~15LL;
    const long long a1 = (b1 + 15) & ~15LL;
    Cover c;
    c.src = reinterpret_cast<const char*>(base) + a0;
    c.bytes = static_cast<unsigned>(a1 - a0);
    c.lead = static_cast<int>((b0 - a0) / static_cast<long long>(sizeof(E)));
    return c;
}

template <class T>
struct Slot
{
    T* diag;               // M + 8 (16-byte covers of position-indexed data: a lead and a tail)
    T* b;                  // M + 8
    unsigned* ent;         // M + 8
    T* val;                // E (chunk entry ranges are whole slices: no cover slack)
    unsigned short* code;  // E
    T* gat;                // Gcap (the last one holds zero: what padding entries read)
};

// Every array's byte size is rounded up to 16 so the next one stays 16-byte aligned.
__host__ __device__ inline size_t r16(size_t b) { return (b + 15) & ~size_t(15); }

template <class T>
__host__ __device__ inline size_t slotBytes(int M, int E, int G)
{
    return 2 * r16(sizeof(T) * (M + 8)) + r16(sizeof(unsigned) * (M + 8)) + r16(sizeof(T) * E) +
           r16(sizeof(unsigned short) * E) + r16(sizeof(T) * G);
}

template <class T>
__host__ __device__ inline size_t gsSmemBytes(int M, int E, int G)
{
    return sizeof(T) * kWin + kStages * slotBytes<T>(M, E, G);
}

template <class T>
__device__ __forceinline__ Slot<T> slotAt(unsigned char* base, int M, int E)
{
    Slot<T> s;
    unsigned char* p = base;
    s.diag = reinterpret_cast<T*>(p); p += r16(sizeof(T) * (M + 8));
    s.b = reinterpret_cast<T*>(p); p += r16(sizeof(T) * (M + 8));
    s.ent = reinterpret_cast<unsigned*>(p); p += r16(sizeof(unsigned) * (M + 8));
    s.val = reinterpret_cast<T*>(p); p += r16(sizeof(T) * E);
    s.code = reinterpret_cast<unsigned short*>(p); p += r16(sizeof(unsigned short) * E);
    s.gat = reinterpret_cast<T*>(p);
    return s;
}

__device__ __forceinline__ ChunkRec loadChunkRec(const int4* __restrict__ recs, int c)
{
    const int4 a = recs[3 * (size_t)c];
    const int4 b = recs[3 * (size_t)c + 1];
    const int4 d = recs[3 * (size_t)c + 2];
    ChunkRec r;
    r.pos0 = a.x; r.m = a.y; r.ent0 = a.z; r.nEnt = a.w;
    r.gat0 = b.x; r.nGat = b.y; r.depth = b.z; r.needUp = b.w;
    r.sameWait = d.x; r.newDepth = d.y; r.pad0 = d.z; r.pad1 = d.w;
    return r;
}

__device__ __forceinline__ unsigned ldAcquireCta(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.cta.shared.u32 %0, [%1];" : "=r"(v) : "r"(smemAddr(p)) : "memory");
    return v;
}
__device__ __forceinline__ void stReleaseCta(unsigned* p, unsigned v)
{
    asm volatile("st.release.cta.shared.u32 [%0], %1;" ::"r"(smemAddr(p)), "r"(v) : "memory");
}
// a barrier among the compute warps only (named barrier 1)
__device__ __forceinline__ void computeSync(int nThreads)
{
    asm volatile("bar.sync 1, %0;" ::"r"(nThreads) : "memory");
}

// Bounded waits: on running out, set the error word; once it is set, give up at once.
__device__ __forceinline__ bool errSet(const int* err) { return *reinterpret_cast<const volatile int*>(err) != 0; }

__device__ __forceinline__ void waitMbar(unsigned long long* b, unsigned parity, int* err)
{
    long long it = 0;
    while (!mbarTryWait(b, parity))
    {
        if ((++it & 255) == 0 && errSet(err)) return;
        if (it > kSpinLimit)
        {
            atomicExch(err, 1);
            return;
        }
    }
}

// wait until the shared word *w >= target
__device__ __forceinline__ void waitShared(const unsigned* w, unsigned target, int* err)
{
    long long it = 0;
    while (ldAcquireCta(w) < target)
    {
        if ((++it & 63) == 0 && errSet(err)) return;
        if (it > kSpinLimit)
        {
            atomicExch(err, 1);
            return;
        }
        __nanosleep(32);
    }
}

// One Gauss-Seidel sweep of one level, in position order. Grid = P parts; blockDim = M + 64:
// M compute threads, then the producer warp, then the service warp.
template <class T>
__global__ void __launch_bounds__(kMaxCompute + 64, 1) gsSweep(GsArgs<T> a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) unsigned long long full[kStages];
    __shared__ __align__(8) unsigned long long empty[kStages];
    __shared__ unsigned chunksDone;   // chunks of this part all compute warps finished (for progress)
    __shared__ unsigned upMin;        // least progress seen among the upstream parts
    const int M = a.maxCells;
    const int E = a.maxEnt;
    T* win = reinterpret_cast<T*>(smem);
    unsigned char* slots = smem + sizeof(T) * kWin;
    const size_t sb = slotBytes<T>(M, E, a.maxGat);
    const int p = blockIdx.x;
    const int t = threadIdx.x;
    const int c0 = a.partChunkStart[p];
    const int nCh = a.partChunkStart[p + 1] - c0;
    const int nComputeWarps = M >> 5;
    if (t < kStages)
    {
        T* g = slotAt<T>(slots + t * sb, M, E).gat;
        g[a.maxGat - 1] = T(0);
    }
    if (t == 0)
    {
        chunksDone = 0u;
        upMin = 0u;
        for (int s = 0; s < kStages; ++s)
        {
            mbarInit(&full[s], 1 + 32);        // the producer's expect_tx + its 32 lanes' gathers
            mbarInit(&empty[s], nComputeWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fenceProxyAsyncShared();
    }
    __syncthreads();
    auto slotOf = [&](int j) { return slotAt<T>(slots + (j % kStages) * sb, M, E); };

    if (t >= M + 32)
    {
        // ---------------- service warp: progress out, upstream progress in ----------------
        const int lane = t - M - 32;
        const int upBeg = a.upStart[p];
        const int upEnd = a.upStart[p + 1];
        const bool publish = a.hasDown[p] != 0;
        unsigned published = 0u;
        if (publish && lane == 0 && nCh > 0)
        {
            published = static_cast<unsigned>(a.chunkRec[3 * (size_t)c0 + 1].z);
            stRelease(&a.progress[p], published);  // nothing of this part lies below its first depth
        }
        long long it = 0;
        unsigned lastDone = 0u;
        while (true)
        {
            // one value for the whole warp: lanes must agree before the shuffles below
            const unsigned done = __shfl_sync(0xffffffffu, ldAcquireCta(&chunksDone), 0);
            if (publish && done != lastDone)
            {
                lastDone = done;
                const unsigned v = done < static_cast<unsigned>(nCh)
                                       ? static_cast<unsigned>(a.chunkRec[3 * (size_t)(c0 + done) + 1].z)
                                       : 0x7fffffffu;
                if (lane == 0 && v > published)
                {
                    __threadfence();
                    stRelease(&a.progress[p], v);
                    published = v;
                }
            }
            if (done >= static_cast<unsigned>(nCh)) break;
            if (upEnd > upBeg)
            {
                unsigned m = 0xffffffffu;
                for (int i = upBeg + lane; i < upEnd; i += 32) m = min(m, ldAcquire(&a.progress[a.upList[i]]));
                for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
                if (lane == 0 && m > ldAcquireCta(&upMin)) stReleaseCta(&upMin, m);
            }
            if (__shfl_sync(0xffffffffu, errSet(a.err) ? 1 : 0, 0)) break;
            if (++it > 16 * kSpinLimit)
            {
                if (lane == 0) atomicExch(a.err, 1);
                break;
            }
            __nanosleep(20);
        }
        return;
    }

    if (t >= M)
    {
        // ---------------- producer warp: stages chunk j into slot j % S ----------------
        const int lane = t - M;
        const int partEnd = a.partPosStart[p + 1];
        const int fillEnd = min(a.nPadded, ((partEnd + kFill - 1) / kFill) * kFill);
        int filled = (a.partPosStart[p] / kFill) * kFill;  // window filled up to here
        // the next chunk's record and first gather sources are loaded a chunk ahead, off the path
        // from a free slot to its copies
        constexpr int kPre = 4;
        ChunkRec nx = nCh > 0 ? loadChunkRec(a.chunkRec, c0) : ChunkRec{};
        int pre[kPre];
#pragma unroll
        for (int k = 0; k < kPre; ++k) pre[k] = (nCh > 0 && lane + 32 * k < nx.nGat) ? a.gatSrc[nx.gat0 + lane + 32 * k] : 0;
        unsigned long long* ptr = a.trace ? a.trace + 4 * (size_t)a.partChunkStart[a.nParts] + 4 * (size_t)a.nParts : nullptr;
        for (int j = 0; j < nCh; ++j)
        {
            const int s = j % kStages;
            const ChunkRec cr = nx;
            int src[kPre];
#pragma unroll
            for (int k = 0; k < kPre; ++k) src[k] = pre[k];
            if (j + 1 < nCh)
            {
                nx = loadChunkRec(a.chunkRec, c0 + j + 1);
#pragma unroll
                for (int k = 0; k < kPre; ++k)
                    pre[k] = lane + 32 * k < nx.nGat ? a.gatSrc[nx.gat0 + lane + 32 * k] : 0;
            }
            if (ptr && lane == 0) ptr[2 * (size_t)(c0 + j)] = clockStamp();
            if (j >= kStages) waitMbar(&empty[s], static_cast<unsigned>((j / kStages - 1) & 1), a.err);
            const Slot<T> sl = slotOf(j);
            if (lane == 0)
            {
                const Cover cd = coverOf(a.posDiag, cr.pos0, cr.m);
                const Cover cbv = coverOf(a.b, cr.pos0, cr.m);
                const Cover cen = coverOf(a.posEnt, cr.pos0, cr.m);
                const unsigned vBytes = static_cast<unsigned>(sizeof(T) * cr.nEnt);
                const unsigned cBytes = static_cast<unsigned>(sizeof(unsigned short) * cr.nEnt);
                const int target = min(fillEnd, ((cr.pos0 + a.ahead + kFill - 1) / kFill) * kFill);
                const int nFill = target > filled ? (target - filled) / kFill : 0;
                const unsigned total = cd.bytes + cbv.bytes + cen.bytes + vBytes + cBytes +
                                       static_cast<unsigned>(nFill) * kFill * sizeof(T);
                mbarExpectTx(&full[s], total);
                tmaLoad(sl.diag, cd.src, cd.bytes, &full[s]);
                tmaLoad(sl.b, cbv.src, cbv.bytes, &full[s]);
                tmaLoad(sl.ent, cen.src, cen.bytes, &full[s]);
                if (cr.nEnt)
                {
                    tmaLoad(sl.val, a.entVal + cr.ent0, vBytes, &full[s]);
                    tmaLoad(sl.code, a.entCode + cr.ent0, cBytes, &full[s]);
                }
                for (int f = 0; f < nFill; ++f, filled += kFill)
                    tmaLoad(win + (filled & (kWin - 1)), a.psi + filled, kFill * sizeof(T), &full[s]);
                // gathered values must be final: owners of other parts once those parts are far
                // enough along, owners of this part once their chunk is consumed (chunk sw is done
                // when empty[sw % S] completes phase sw / S; the wait for slot j - S above already
                // covers every chunk up to j - S, and phase sw / S + 1 needs chunk sw + S > j, so
                // the parity is unambiguous)
                if (cr.needUp >= 0) waitShared(&upMin, static_cast<unsigned>(cr.needUp) + 1u, a.err);
                const int sw = cr.sameWait - c0;
                if (cr.sameWait >= 0 && sw > j - kStages)
                    waitMbar(&empty[sw % kStages], static_cast<unsigned>((sw / kStages) & 1), a.err);
            }
            __syncwarp();
#pragma unroll
            for (int k = 0; k < kPre; ++k)
                if (lane + 32 * k < cr.nGat) __pipeline_memcpy_async(&sl.gat[lane + 32 * k], &a.psi[src[k]], sizeof(T));
            for (int g = lane + 32 * kPre; g < cr.nGat; g += 32)
                __pipeline_memcpy_async(&sl.gat[g], &a.psi[a.gatSrc[cr.gat0 + g]], sizeof(T));
            mbarArriveCpAsync(&full[s]);
            if (ptr && lane == 0) ptr[2 * (size_t)(c0 + j) + 1] = clockStamp();
        }
        return;
    }

    // ---------------- compute warps: one thread per cell ----------------
    const int lane = t & 31;
    unsigned long long* ptrace = a.trace ? a.trace + 4 * (size_t)a.partChunkStart[a.nParts] + 4 * (size_t)p : nullptr;
    if (ptrace && t == 0)
    {
        ptrace[0] = globalTimer();
        ptrace[1] = clockStamp();
    }
    // 32-bit shared addresses: the window, and slot 0's arrays (slot s is sb bytes further on)
    const unsigned winA = smemAddr(win);
    const Slot<T> s0 = slotAt<T>(slots, M, E);
    const unsigned diagA = smemAddr(s0.diag), bA = smemAddr(s0.b), entA = smemAddr(s0.ent);
    const unsigned valA = smemAddr(s0.val), codeA = smemAddr(s0.code), gatA = smemAddr(s0.gat);
    const unsigned sb32 = static_cast<unsigned>(sb);
    constexpr unsigned kT = sizeof(T);
    ChunkRec nx = nCh > 0 ? loadChunkRec(a.chunkRec, c0) : ChunkRec{};
    int s = 0;
    unsigned phase = 0u;
    for (int j = 0; j < nCh; ++j)
    {
        const ChunkRec cr = nx;
        if (j + 1 < nCh) nx = loadChunkRec(a.chunkRec, c0 + j + 1);
        if (a.trace && t == 0) a.trace[4 * (size_t)(c0 + j)] = clockStamp();
        if (cr.newDepth && j > 0)
        {
            // the owners this chunk reads were computed by any compute warp: wait for all of them
            computeSync(M);
            if (t == 0) stReleaseCta(&chunksDone, static_cast<unsigned>(j));
        }
        waitMbar(&full[s], phase, a.err);
        if (a.trace && t == 0) a.trace[4 * (size_t)(c0 + j) + 1] = clockStamp();
        if (t < cr.m)
        {
            const unsigned so = static_cast<unsigned>(s) * sb32;
            // leads of the 16-byte covers the producer copied (diagonal and b: T; descriptors: u32)
            const unsigned lT = (static_cast<unsigned>(cr.pos0) * kT & 15u) / kT;
            const unsigned lE = static_cast<unsigned>(cr.pos0) & 3u;
            const unsigned pe = ldsU32(entA + so + 4u * (lE + t));
            T acc = ldsT(bA + so + kT * (lT + t), T());
            const T dg = ldsT(diagA + so + kT * (lT + t), T());
            const int width = static_cast<int>(pe >> 24);
            const unsigned rb = pe & 0xffffffu;
            const unsigned cA = codeA + so + 2u * rb;
            const unsigned vA = valA + so + kT * rb;
            const unsigned gA = gatA + so;
            constexpr int kRegs = 8;
            for (int q0 = 0; q0 < width; q0 += kRegs)
            {
                // width is the same for the whole warp: these branches do not diverge
                unsigned c[kRegs];
                T w[kRegs], v[kRegs];
#pragma unroll
                for (int q = 0; q < kRegs; ++q)
                    if (q0 + q < width)
                    {
                        c[q] = ldsU16(cA + 64u * (q0 + q));
                        w[q] = ldsT(vA + 32u * kT * (q0 + q), T());
                    }
#pragma unroll
                for (int q = 0; q < kRegs; ++q)
                    if (q0 + q < width)
                        v[q] = ldsT((c[q] & kGatBit) ? gA + kT * (c[q] & (kGatBit - 1u)) : winA + kT * c[q], T());
#pragma unroll
                for (int q = 0; q < kRegs; ++q)
                    if (q0 + q < width) acc = subRn(acc, mulRn(w[q], v[q]));
            }
            const T res = divRn(acc, dg);
            const int pos = cr.pos0 + t;
            stsT(winA + kT * static_cast<unsigned>(pos & (kWin - 1)), res);
            // this window slot is refilled by TMA (the async proxy) one window later; the fence comes
            // before the global store so that it does not wait for that store
            fenceProxyAsyncShared();
            a.psi[pos] = res;
        }
        if (a.trace && t == 0) a.trace[4 * (size_t)(c0 + j) + 2] = clockStamp();
        __syncwarp();
        if (lane == 0) mbarArrive(&empty[s]);
        if (a.trace && t == 0) a.trace[4 * (size_t)(c0 + j) + 3] = clockStamp();
        if (++s == kStages)
        {
            s = 0;
            phase ^= 1u;
        }
    }
    computeSync(M);
    if (t == 0) stReleaseCta(&chunksDone, static_cast<unsigned>(nCh));
    if (ptrace && t == 0)
    {
        ptrace[2] = globalTimer();
        ptrace[3] = clockStamp();
    }
}

}  // namespace k
}  // namespace b2g
