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
// THE SCHEDULE (part-pipelined, one sweep per launch). Cells are split into P contiguous index
// ranges ("parts"), one persistent CTA per part. A part's cells are laid out by (depth, cell) and cut
// into "chunks" of at most M cells of one depth, walked in order.
//
// WARP ROLES. The compute warps run the chunks through an S-slot shared-memory pipeline: a chunk's
// contiguous data (cell ids, row offsets, diagonal, entry codes and coefficients, all in position
// order) is copied with cp.async S-1 chunks ahead; G chunks ahead, once its codes have landed, the
// gathers it needs that are already final are issued too (b, and kind PRE: old values of upper
// neighbours, and owners two or more chunks back). Owners the part computed within the last R
// positions come from a shared-memory ring (kind RING). Only owners held by other parts (and rare
// far owners one chunk back) are read from global memory at compute time (kind LATE). The service
// warp takes the two global-memory handshakes off the compute path: it publishes the part's
// progress word ("every cell of depth < d is done", release at GPU scope) whenever the compute warps
// report a finished depth through shared memory, and it polls the upstream parts' words and posts
// their minimum in shared memory, which the compute warps check before a chunk with LATE owners.
//
// WHY PRE IS SAFE. An upper neighbour n of a cell c has depth(n) > depth(c), so n is rewritten only
// after c's depth completes: in this part after c's chunk, in another part only after that part saw
// this part's progress pass depth(c), which is published after c's chunk. c's gathers are issued
// before c's chunk runs.
//
// BOUNDED WAITS. Every spin has a budget; when it runs out the error word is set and every later wait
// returns at once, so a broken schedule ends the kernel with an error instead of hanging the GPU.
#pragma once

#include <cuda_pipeline.h>

#include "b2g_common.cuh"

namespace b2g {
namespace k {

constexpr int kRingLog = 12;
constexpr int kRing = 1 << kRingLog;           // shared-memory ring of recent values (positions)
constexpr unsigned kKindShift = 30;
constexpr unsigned kIdxMask = (1u << kKindShift) - 1u;
enum : unsigned { KIND_RING = 0u, KIND_PRE = 1u, KIND_LATE = 2u };
constexpr int kStages = 6;                     // S: pipeline slots
constexpr int kGatherAhead = 2;                // G: chunks ahead the gathers are issued (S >= G + 2)
constexpr int kRowRegs = 8;                    // row entries resolved into registers before the chain
constexpr long long kSpinLimit = 1LL << 24;    // polls before a wait gives up (~1-2 s with backoff)

template <class T>
struct GsArgs
{
    int nParts;
    int maxCells;                  // M: chunk cell capacity (compute threads)
    int maxEnt;                    // E: chunk entry capacity
    const int* __restrict__ partChunkStart;  // [P+1]
    const int4* __restrict__ chunkRec;       // [nChunks][2]: {pos0, m, e0, ne}, {depth, needUp, -, -}
    const int* __restrict__ upStart;         // [P+1]
    const int* __restrict__ upList;
    const int* __restrict__ hasDown;         // [P] 1 if another part reads this part's values
    const int* __restrict__ posCell;         // [n]
    const int* __restrict__ posRow;          // [n+1] entry offsets in position order
    const unsigned* __restrict__ entCode;    // [nnz] kind << 30 | index (ring slot or cell)
    const T* __restrict__ entVal;            // [nnz]
    const T* __restrict__ posDiag;           // [n]
    const T* __restrict__ b;                 // by cell
    T* psi;                                  // by cell, updated in place
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

template <class T>
struct Slot
{
    T* diag;
    T* b;
    T* val;
    T* old;
    int* cell;
    int* row;        // M + 1 absolute entry offsets
    unsigned* code;
};

template <class T>
__host__ __device__ inline size_t slotBytes(int M, int E)
{
    const size_t b = 2 * sizeof(T) * M + 2 * sizeof(T) * E + sizeof(int) * M + sizeof(int) * (M + 1) +
                     sizeof(unsigned) * E;
    return (b + 15) & ~size_t(15);
}

template <class T>
__host__ __device__ inline size_t gsSmemBytes(int M, int E)
{
    return sizeof(T) * kRing + kStages * slotBytes<T>(M, E);
}

template <class T>
__device__ __forceinline__ Slot<T> slotAt(unsigned char* base, int M, int E)
{
    Slot<T> s;
    unsigned char* p = base;
    s.diag = reinterpret_cast<T*>(p); p += sizeof(T) * M;
    s.b = reinterpret_cast<T*>(p); p += sizeof(T) * M;
    s.val = reinterpret_cast<T*>(p); p += sizeof(T) * E;
    s.old = reinterpret_cast<T*>(p); p += sizeof(T) * E;
    s.cell = reinterpret_cast<int*>(p); p += sizeof(int) * M;
    s.row = reinterpret_cast<int*>(p); p += sizeof(int) * (M + 1);
    s.code = reinterpret_cast<unsigned*>(p);
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
    asm volatile("ld.acquire.cta.shared.u32 %0, [%1];"
                 : "=r"(v)
                 : "r"(static_cast<unsigned>(__cvta_generic_to_shared(p)))
                 : "memory");
    return v;
}
__device__ __forceinline__ void stReleaseCta(unsigned* p, unsigned v)
{
    asm volatile("st.release.cta.shared.u32 [%0], %1;" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(p))),
                 "r"(v)
                 : "memory");
}
// a barrier among the compute warps only (named barrier 1)
__device__ __forceinline__ void computeSync(int nThreads)
{
    asm volatile("bar.sync 1, %0;" ::"r"(nThreads) : "memory");
}

// One Gauss-Seidel sweep of one level. Grid = P parts; blockDim = M compute threads + 32.
template <class T>
__global__ void __launch_bounds__(512) gsSweep(GsArgs<T> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ ChunkRec rec[kStages];
    __shared__ unsigned chunksDone;   // chunks of this part the compute warps have finished
    __shared__ unsigned upMin;        // least progress seen among the upstream parts
    const int M = a.maxCells;
    const int E = a.maxEnt;
    T* ring = reinterpret_cast<T*>(smem);
    const size_t sb = slotBytes<T>(M, E);
    const int p = blockIdx.x;
    const int t = threadIdx.x;
    const int c0 = a.partChunkStart[p];
    const int nCh = a.partChunkStart[p + 1] - c0;
    if (t == 0)
    {
        chunksDone = 0u;
        upMin = 0u;
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
    unsigned char* slots = smem + sizeof(T) * kRing;
    auto slotOf = [&](int j) { return slotAt<T>(slots + (j % kStages) * sb, M, E); };
    // records of the next two chunks to stage, loaded ahead (no dependent loads on the loop)
    ChunkRec rq0 = loadChunkRec(a.chunkRec, c0, 0 < nCh);
    ChunkRec rq1 = loadChunkRec(a.chunkRec, c0 + 1, 1 < nCh);
    unsigned long long* ptrace = a.trace ? a.trace + 4 * (size_t)a.partChunkStart[a.nParts] + 4 * (size_t)p : nullptr;
    if (ptrace && t == 0)
    {
        ptrace[0] = globalTimer();
        ptrace[1] = clock64();
    }
    for (int r = -(kStages - 1); r < nCh; ++r)
    {
        if (a.trace && t == 0 && r >= 0) a.trace[4 * (size_t)(c0 + r)] = clock64();
        // (1) chunk r+G's codes have landed (and chunk r-1 is written: this barrier also ends it)
        __pipeline_wait_prior(kStages - kGatherAhead - 2);
        computeSync(M);
        if (a.trace && t == 0 && r >= 0) a.trace[4 * (size_t)(c0 + r) + 1] = clock64();
        if (t == 0 && r >= 1) stReleaseCta(&chunksDone, static_cast<unsigned>(r));
        // (2) contiguous stage of chunk r+S-1 into the slot chunk r-1 released
        const int jc = r + kStages - 1;
        if (jc < nCh)
        {
            const Slot<T> s = slotOf(jc);
            const ChunkRec cr = rq0;
            if (t == 0) rec[jc % kStages] = cr;
            for (int i = t; i < cr.m; i += M)
            {
                __pipeline_memcpy_async(&s.cell[i], &a.posCell[cr.pos0 + i], sizeof(int));
                __pipeline_memcpy_async(&s.diag[i], &a.posDiag[cr.pos0 + i], sizeof(T));
                __pipeline_memcpy_async(&s.row[i], &a.posRow[cr.pos0 + i], sizeof(int));
            }
            if (t == 0) __pipeline_memcpy_async(&s.row[cr.m], &a.posRow[cr.pos0 + cr.m], sizeof(int));
            for (int e = t; e < cr.ne; e += M)
            {
                __pipeline_memcpy_async(&s.code[e], &a.entCode[cr.e0 + e], sizeof(unsigned));
                __pipeline_memcpy_async(&s.val[e], &a.entVal[cr.e0 + e], sizeof(T));
            }
            rq0 = rq1;
            rq1 = loadChunkRec(a.chunkRec, c0 + jc + 2, jc + 2 < nCh);
        }
        // (3) gathers of chunk r+G: b, and every value already final
        const int jg = r + kGatherAhead;
        if (jg >= 0 && jg < nCh)
        {
            const Slot<T> s = slotOf(jg);
            const ChunkRec& gr = rec[jg % kStages];
            for (int i = t; i < gr.m; i += M) __pipeline_memcpy_async(&s.b[i], &a.b[s.cell[i]], sizeof(T));
            for (int e = t; e < gr.ne; e += M)
            {
                const unsigned c = s.code[e];
                if ((c >> kKindShift) == KIND_PRE)
                    __pipeline_memcpy_async(&s.old[e], &a.psi[c & kIdxMask], sizeof(T));
            }
        }
        __pipeline_commit();
        if (r < 0) continue;
        // (4) chunk r's data in place; the parts holding its LATE owners far enough along
        __pipeline_wait_prior(kGatherAhead);
        const ChunkRec& cr = rec[r % kStages];
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
        if (a.trace && t == 0) a.trace[4 * (size_t)(c0 + r) + 2] = clock64();
        // (5) the sweep: resolve the row's values first, then the reference's rounding chain
        const Slot<T> s = slotOf(r);
        if (t < cr.m)
        {
            const int rb = s.row[t] - cr.e0;
            const int re = s.row[t + 1] - cr.e0;
            T acc = s.b[t];
            for (int e0 = rb; e0 < re; e0 += kRowRegs)
            {
                T v[kRowRegs], w[kRowRegs];
#pragma unroll
                for (int q = 0; q < kRowRegs; ++q)
                {
                    const int e = e0 + q;
                    if (e < re)
                    {
                        const unsigned c = s.code[e];
                        const unsigned kind = c >> kKindShift;
                        const unsigned idx = c & kIdxMask;
                        w[q] = s.val[e];
                        v[q] = kind == KIND_RING ? ring[idx] : (kind == KIND_PRE ? s.old[e] : ldcg(&a.psi[idx]));
                    }
                }
#pragma unroll
                for (int q = 0; q < kRowRegs; ++q)
                    if (e0 + q < re) acc = subRn(acc, mulRn(w[q], v[q]));
            }
            const T res = divRn(acc, s.diag[t]);
            a.psi[s.cell[t]] = res;
            ring[(cr.pos0 + t) & (kRing - 1)] = res;
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
