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
// its positions in order, cut into "chunks" of at most M cells of one depth.
//
// WHAT A CHUNK READS, AND FROM WHERE.
//   * Its contiguous data -- diagonal, b, row offsets, entry codes, coefficients -- is copied into
//     one of S shared-memory slots by TMA bulk copies (cp.async.bulk + mbarrier), S-1 chunks ahead.
//   * psi itself lives, around the sweep front, in a shared-memory window of W positions: behind the
//     front the part's NEW values (written as they are computed), ahead of it the OLD values,
//     streamed in by TMA bulk copies as the front advances. Entry kind WIN reads the window.
//   * What the window does not hold is gathered G chunks ahead (kind GAT): old values of
//     neighbours outside the window or in other parts, owners computed long enough ago, and owners
//     held by other parts -- those only once the upstream parts' progress covers them (else at
//     compute time, after the wait). Kind SLOW (an owner just outside the window, computed too
//     recently to gather ahead) is read at compute time.
//
// WARP ROLES. Compute warps run the chunks; one service warp publishes the part's progress word
// ("every cell of depth < d is done", release at GPU scope) when the compute warps report a depth
// through shared memory, and polls the upstream parts' words, posting their minimum in shared
// memory for the compute warps.
//
// WHY OLD VALUES MAY BE READ EARLY. A neighbour n of a cell c has depth(n) > depth(c), so n is
// rewritten only after c's depth completes: in this part after c's chunk, in another part only after
// that part saw this part's progress pass depth(c), which is published after c's chunk.
//
// BOUNDED WAITS. Every spin has a budget; when it runs out the error word is set and every later wait
// returns at once, so a broken schedule ends the kernel with an error instead of hanging the GPU.
#pragma once

#include <cuda_pipeline.h>

#include "b2g_common.cuh"

namespace b2g {
namespace k {

constexpr int kWin = 4096;                     // W: psi window (positions), a power of two
constexpr int kFill = 256;                     // B: window fill block (positions)
constexpr unsigned kKindShift = 30;
constexpr unsigned kIdxMask = (1u << kKindShift) - 1u;
enum : unsigned { KIND_WIN = 0u, KIND_GAT = 1u, KIND_SLOW = 2u };
constexpr int kStages = 6;                     // S: pipeline slots
constexpr int kGatherAhead = 2;                // G: chunks ahead the gathers are issued
constexpr long long kSpinLimit = 1LL << 24;    // polls before a wait gives up (~1-2 s with backoff)

// Window extents the schedule guarantees for a chunk starting at s and ending at e: positions
// [s, s + ahead) hold old values, [e - behind, s) new ones. The fills issued S-1 chunks ahead must
// not overwrite new values a pending chunk still reads, hence ahead + behind + B + (S-2)*M <= W.
inline void gsWindowExtents(int M, int& ahead, int& behind)
{
    const int room = kWin - kFill - (kStages - 2) * M;
    ahead = room / 2;
    behind = room - ahead;
}

template <class T>
struct GsArgs
{
    int nParts;
    int maxCells;                  // M: chunk cell capacity (compute threads)
    int maxEnt;                    // E: chunk entry capacity
    int ahead;                     // window extent ahead of a chunk's start (positions)
    int nPadded;                   // psi / b / diag arrays are readable up to here (fill blocks)
    const int* __restrict__ partChunkStart;  // [P+1]
    const int* __restrict__ partPosStart;    // [P+1]
    const int4* __restrict__ chunkRec;       // [nChunks][2]: {pos0, m, e0, ne}, {depth, needUp, -, -}
    const int* __restrict__ upStart;         // [P+1]
    const int* __restrict__ upList;
    const int* __restrict__ hasDown;         // [P] 1 if another part reads this part's values
    const int* __restrict__ posRow;          // [n+1] entry offsets in position order (padded)
    const unsigned* __restrict__ entCode;    // [nnz] kind << 30 | window slot or position (padded)
    const T* __restrict__ entVal;            // [nnz] (padded)
    const T* __restrict__ posDiag;           // [n] (padded)
    const T* __restrict__ b;                 // [n] by position (padded)
    T* psi;                                  // [n] by position, updated in place (padded)
    unsigned* progress;                      // [P]
    int* err;
    unsigned long long* trace;               // diagnostic: [nChunks][4] clock64 stamps + [P][4] part
                                             // {globaltimer, clock64} at start and end, or null
};

__device__ __forceinline__ unsigned long long globalTimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
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
    T* diag;        // M + 8
    T* b;           // M + 8
    T* val;         // E + 8
    T* gat;         // E      (gathered values, by entry)
    int* row;       // M + 9
    unsigned* code; // E + 8
};

// Each TMA destination holds its elements plus up to 8 of cover rounding; every array's byte size
// is rounded up to 16 so the next one stays 16-byte aligned.
__host__ __device__ inline size_t r16(size_t b) { return (b + 15) & ~size_t(15); }

template <class T>
__host__ __device__ inline size_t slotBytes(int M, int E)
{
    return 2 * r16(sizeof(T) * (M + 8)) + r16(sizeof(T) * (E + 8)) + r16(sizeof(int) * (M + 9)) +
           r16(sizeof(unsigned) * (E + 8)) + r16(sizeof(T) * E);
}

template <class T>
__host__ __device__ inline size_t gsSmemBytes(int M, int E)
{
    return sizeof(T) * kWin + kStages * slotBytes<T>(M, E);
}

template <class T>
__device__ __forceinline__ Slot<T> slotAt(unsigned char* base, int M, int E)
{
    Slot<T> s;
    unsigned char* p = base;
    s.diag = reinterpret_cast<T*>(p); p += r16(sizeof(T) * (M + 8));
    s.b = reinterpret_cast<T*>(p); p += r16(sizeof(T) * (M + 8));
    s.val = reinterpret_cast<T*>(p); p += r16(sizeof(T) * (E + 8));
    s.row = reinterpret_cast<int*>(p); p += r16(sizeof(int) * (M + 9));
    s.code = reinterpret_cast<unsigned*>(p); p += r16(sizeof(unsigned) * (E + 8));
    s.gat = reinterpret_cast<T*>(p);
    return s;
}

struct ChunkRec
{
    int pos0, m, e0, ne, depth, needUp;
};

__device__ __forceinline__ ChunkRec loadChunkRec(const int4* __restrict__ recs, int c, bool valid)
{
    ChunkRec r;
    if (valid)
    {
        const int4 a = recs[2 * (size_t)c];
        const int4 b = recs[2 * (size_t)c + 1];
        r.pos0 = a.x; r.m = a.y; r.e0 = a.z; r.ne = a.w; r.depth = b.x; r.needUp = b.y;
    }
    else
    {
        r.pos0 = r.m = r.e0 = r.ne = r.depth = 0;
        r.needUp = -1;
    }
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

__device__ __forceinline__ void waitMbar(unsigned long long* b, unsigned parity, int* err)
{
    long long it = 0;
    while (!mbarTryWait(b, parity))
    {
        if (++it > kSpinLimit)
        {
            atomicExch(err, 1);
            break;
        }
    }
}

// One Gauss-Seidel sweep of one level, in position order. Grid = P parts; blockDim = M + 32.
template <class T>
__global__ void __launch_bounds__(512) gsSweep(GsArgs<T> a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ ChunkRec rec[kStages];
    __shared__ int gatherEarly[kStages];          // the chunk's gathers were issued ahead
    __shared__ __align__(8) unsigned long long bar[kStages];
    __shared__ unsigned chunksDone;               // chunks of this part the compute warps finished
    __shared__ unsigned upMin;                    // least progress seen among the upstream parts
    const int M = a.maxCells;
    const int E = a.maxEnt;
    T* win = reinterpret_cast<T*>(smem);
    unsigned char* slots = smem + sizeof(T) * kWin;
    const size_t sb = slotBytes<T>(M, E);
    const int p = blockIdx.x;
    const int t = threadIdx.x;
    const int c0 = a.partChunkStart[p];
    const int nCh = a.partChunkStart[p + 1] - c0;
    if (t == 0)
    {
        chunksDone = 0u;
        upMin = 0u;
        for (int s = 0; s < kStages; ++s) mbarInit(&bar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();

    if (t >= M)
    {
        // ---------------- service warp ----------------
        const int lane = t - M;
        const int upBeg = a.upStart[p];
        const int upEnd = a.upStart[p + 1];
        const bool publish = a.hasDown[p] != 0;
        unsigned published = 0u;
        if (publish && lane == 0 && nCh > 0)
        {
            published = static_cast<unsigned>(a.chunkRec[2 * (size_t)c0 + 1].x);
            stRelease(&a.progress[p], published);  // nothing of this part lies above its first depth
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
                                       ? static_cast<unsigned>(a.chunkRec[2 * (size_t)(c0 + done) + 1].x)
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
            if (__shfl_sync(0xffffffffu, *reinterpret_cast<volatile int*>(a.err), 0)) break;
            if (++it > 16 * kSpinLimit)
            {
                if (lane == 0) atomicExch(a.err, 1);
                break;
            }
            __nanosleep(20);
        }
        return;
    }

    // ---------------- compute warps ----------------
    auto slotOf = [&](int j) { return slotAt<T>(slots + (j % kStages) * sb, M, E); };
    const int partEnd = a.partPosStart[p + 1];
    const int fillEnd = min(a.nPadded, ((partEnd + kFill - 1) / kFill) * kFill);
    int filled = (a.partPosStart[p] / kFill) * kFill;  // window filled up to here (thread 0's view)
    unsigned long long* ptrace = a.trace ? a.trace + 4 * (size_t)a.partChunkStart[a.nParts] + 4 * (size_t)p : nullptr;
    if (ptrace && t == 0)
    {
        ptrace[0] = globalTimer();
        ptrace[1] = clock64();
    }
    ChunkRec rq0 = loadChunkRec(a.chunkRec, c0, 0 < nCh);
    ChunkRec rq1 = loadChunkRec(a.chunkRec, c0 + 1, 1 < nCh);
    for (int r = -(kStages - 1); r < nCh; ++r)
    {
        if (a.trace && t == 0 && r >= 0) a.trace[4 * (size_t)(c0 + r)] = clock64();
        // (1) chunk r+G's data has landed: its gathers can be issued
        const int jg = r + kGatherAhead;
        if (jg >= 0 && jg < nCh)
        {
            waitMbar(&bar[jg % kStages], static_cast<unsigned>((jg / kStages) & 1), a.err);
            if (t == 0)
            {
                const int nu = rec[jg % kStages].needUp;
                gatherEarly[jg % kStages] =
                    (nu < 0 || ldAcquireCta(&upMin) >= static_cast<unsigned>(nu) + 1u) ? 1 : 0;
            }
        }
        computeSync(M);  // also: chunk r-1 is complete and its slot free
        if (a.trace && t == 0 && r >= 0) a.trace[4 * (size_t)(c0 + r) + 1] = clock64();
        if (t == 0 && r >= 1) stReleaseCta(&chunksDone, static_cast<unsigned>(r));
        // (2) chunk r+S-1: its contiguous data and the window's old values it needs, by TMA
        const int jc = r + kStages - 1;
        if (jc < nCh)
        {
            if (t == 0)
            {
                const Slot<T> s = slotOf(jc);
                const ChunkRec cr = rq0;
                rec[jc % kStages] = cr;
                const Cover cd = coverOf(a.posDiag, cr.pos0, cr.m);
                const Cover cbv = coverOf(a.b, cr.pos0, cr.m);
                const Cover cro = coverOf(a.posRow, cr.pos0, cr.m + 1);
                const Cover cco = coverOf(a.entCode, cr.e0, cr.ne);
                const Cover cva = coverOf(a.entVal, cr.e0, cr.ne);
                const int target = min(fillEnd, ((cr.pos0 + a.ahead + kFill - 1) / kFill) * kFill);
                const int nFill = target > filled ? (target - filled) / kFill : 0;
                const unsigned total = cd.bytes + cbv.bytes + cro.bytes + (cr.ne ? cco.bytes + cva.bytes : 0u) +
                                       static_cast<unsigned>(nFill) * kFill * sizeof(T);
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                unsigned long long* b = &bar[jc % kStages];
                mbarExpectTx(b, total);
                tmaLoad(s.diag, cd.src, cd.bytes, b);
                tmaLoad(s.b, cbv.src, cbv.bytes, b);
                tmaLoad(s.row, cro.src, cro.bytes, b);
                if (cr.ne)
                {
                    tmaLoad(s.code, cco.src, cco.bytes, b);
                    tmaLoad(s.val, cva.src, cva.bytes, b);
                }
                for (int f = 0; f < nFill; ++f, filled += kFill)
                    tmaLoad(win + (filled & (kWin - 1)), a.psi + filled, kFill * sizeof(T), b);
            }
            rq0 = rq1;
            rq1 = loadChunkRec(a.chunkRec, c0 + jc + 2, jc + 2 < nCh);
        }
        // (3) chunk r+G's gathers, when everything they read is final
        if (jg >= 0 && jg < nCh && gatherEarly[jg % kStages])
        {
            const Slot<T> s = slotOf(jg);
            const ChunkRec& gr = rec[jg % kStages];
            const int lc = coverOf(a.entCode, gr.e0, gr.ne).lead;
            for (int e = t; e < gr.ne; e += M)
            {
                const unsigned c = s.code[lc + e];
                if ((c >> kKindShift) == KIND_GAT) __pipeline_memcpy_async(&s.gat[e], &a.psi[c & kIdxMask], sizeof(T));
            }
        }
        __pipeline_commit();
        if (r < 0) continue;
        // (4) chunk r: its data, its gathers, and the parts holding its owners far enough along
        __pipeline_wait_prior(kGatherAhead);
        const ChunkRec cr = rec[r % kStages];
        waitMbar(&bar[r % kStages], static_cast<unsigned>((r / kStages) & 1), a.err);
        const bool early = gatherEarly[r % kStages] != 0;
        if (t == 0 && cr.needUp >= 0)
        {
            const unsigned target = static_cast<unsigned>(cr.needUp) + 1u;
            long long it = 0;
            while (ldAcquireCta(&upMin) < target)
            {
                if (*reinterpret_cast<volatile int*>(a.err)) break;
                if (++it > kSpinLimit)
                {
                    atomicExch(a.err, 1);
                    break;
                }
                __nanosleep(16);
            }
        }
        computeSync(M);
        const Slot<T> s = slotOf(r);
        const int lc = coverOf(a.entCode, cr.e0, cr.ne).lead;
        const int lv = coverOf(a.entVal, cr.e0, cr.ne).lead;
        if (!early)
        {
            // the upstream parts were not far enough along when the gathers were due
            for (int e = t; e < cr.ne; e += M)
            {
                const unsigned c = s.code[lc + e];
                if ((c >> kKindShift) == KIND_GAT) s.gat[e] = ldcg(&a.psi[c & kIdxMask]);
            }
            computeSync(M);
        }
        if (a.trace && t == 0) a.trace[4 * (size_t)(c0 + r) + 2] = clock64();
        // (5) the sweep: the row's values first, then the reference's rounding chain
        if (t < cr.m)
        {
            const int ld = coverOf(a.posDiag, cr.pos0, cr.m).lead;
            const int lb = coverOf(a.b, cr.pos0, cr.m).lead;
            const int lr = coverOf(a.posRow, cr.pos0, cr.m + 1).lead;
            const int rb = s.row[lr + t] - cr.e0;
            const int re = s.row[lr + t + 1] - cr.e0;
            T acc = s.b[lb + t];
            constexpr int kRegs = 8;
            for (int e0 = rb; e0 < re; e0 += kRegs)
            {
                T v[kRegs], w[kRegs];
#pragma unroll
                for (int q = 0; q < kRegs; ++q)
                {
                    const int e = e0 + q;
                    if (e < re)
                    {
                        const unsigned c = s.code[lc + e];
                        const unsigned kind = c >> kKindShift;
                        const unsigned idx = c & kIdxMask;
                        w[q] = s.val[lv + e];
                        v[q] = kind == KIND_WIN ? win[idx] : (kind == KIND_GAT ? s.gat[e] : ldcg(&a.psi[idx]));
                    }
                }
#pragma unroll
                for (int q = 0; q < kRegs; ++q)
                    if (e0 + q < re) acc = subRn(acc, mulRn(w[q], v[q]));
            }
            const T res = divRn(acc, s.diag[ld + t]);
            const int pos = cr.pos0 + t;
            a.psi[pos] = res;
            win[pos & (kWin - 1)] = res;
        }
        if (a.trace && t == 0) a.trace[4 * (size_t)(c0 + r) + 3] = clock64();
    }
    __pipeline_wait_prior(0);
    computeSync(M);
    if (t == 0) stReleaseCta(&chunksDone, static_cast<unsigned>(nCh));
    if (ptrace && t == 0)
    {
        ptrace[2] = globalTimer();
        ptrace[3] = clock64();
    }
}

}  // namespace k
}  // namespace b2g
