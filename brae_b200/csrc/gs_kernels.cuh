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
// THE CRITICAL PATH. A sweep takes about (DAG depth) x (time per chunk), and a chunk's time is the
// instruction stream of its rows (a lone warp issues about one instruction per 5 cycles of this
// code), so everything but the row arithmetic is taken off the compute warps, and a row entry is
// reduced to three loads (code, coefficient, value), a multiply and a subtraction:
//   * a PRODUCER warp stages chunk j, S-1 chunks ahead, into one of S shared-memory slots: the
//     chunk's blob (diagonal, row descriptors, coefficients, codes -- one contiguous TMA bulk copy)
//     and b (a second one), the psi window's old values ahead of the front (TMA), and by cp.async
//     the values the window does not hold; all of it completes on the slot's `full` mbarrier;
//   * a PUBLISHER warp releases the part's progress word as the compute warps pass each depth, and
//     a WATCHER warp polls the upstream parts' words;
//   * the COMPUTE warps (one thread per cell) wait on `full`, compute their rows from shared
//     memory only, and release the slot warp by warp on its `empty` mbarrier.
//
// THE VALUE TABLE. One shared-memory array holds every value a row reads: [0, W) the psi window,
// [W + s*G, W + (s+1)*G) the values gathered for the chunk in stage s, and W + S*G a zero. An entry
// code is the 16-bit index of its value in the table: the schedule knows each chunk's stage (the
// chunk's index in its part, mod S), so no code needs decoding.
//
// ENTRY LAYOUT (sliced ELL, per chunk). A chunk's entries are stored in slices of 32 cells (one
// warp): entry q of the cell in lane l of a slice sits at sliceBase + 32*q + l, so a warp reads 32
// consecutive codes and coefficients per entry -- free of shared-memory bank conflicts. A cell's
// row descriptor is width << 24 | (its slice base + lane, relative to the chunk), the width being
// the slice's longest row: every lane of a warp walks the same number of entries, the shorter rows
// padded with entries that read the zero with coefficient zero (acc - 0*0 == acc, so the padding
// leaves the result bit for bit as it is).
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

#include "b2g_common.cuh"

namespace b2g {
namespace k {

constexpr int kWin = 4096;                     // W: psi window (positions), a power of two
constexpr int kFill = 256;                     // B: window fill block (positions)
constexpr int kStages = 4;                     // S: pipeline slots
constexpr int kMaxTable = 65535;               // value-table entries a 16-bit code can name
constexpr int kMaxCompute = 384;               // compute threads per CTA, at most (+ 4 warps)
constexpr long long kSpinLimit = 1LL << 24;    // polls before a wait gives up (the default)
constexpr int kProgressStride = 32;            // progress words 128 bytes apart: one L2 line per part,
                                               // so that a part's publishes meet only its own pollers

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

__host__ __device__ inline unsigned r16(unsigned b) { return (b + 15u) & ~15u; }

// A chunk's blob: [diagonal: m T][row descriptors: m u32]([storage positions: m u32])[coefficients:
// nEnt T][codes: nEnt u16], each part starting 16-byte aligned (nEnt is a multiple of 32). The
// storage positions are there only in an item schedule (several sweeps pipelined, below), whose
// window slots index items, not the psi positions they write.
struct BlobLayout
{
    unsigned desc, store, val, code, bytes;
};
template <class T>
__host__ __device__ inline BlobLayout blobLayout(int m, int nEnt, int items = 0)
{
    BlobLayout L;
    L.desc = r16(static_cast<unsigned>(sizeof(T)) * m);
    L.store = L.desc + r16(4u * m);
    L.val = items ? L.store + r16(4u * m) : L.store;
    L.code = L.val + static_cast<unsigned>(sizeof(T)) * nEnt;
    L.bytes = L.code + r16(2u * nEnt);
    return L;
}

// Chunk record, 12 ints (three int4).
struct ChunkRec
{
    int pos0, m, ent0, nEnt;        // positions [pos0, pos0+m); ELL entries [ent0, ent0+nEnt)
    int gat0, nGat, depth, needUp;  // gather list [gat0, gat0+nGat); other-part owners' max depth or -1
    int sameWait;                   // last same-part chunk a gather reads (global index) or -1
    int newDepth, nOld;             // stored as newDepth | nOld << 1: 1 where the depth changes within
                                    // the part; the gather list's leading old values (final already)
    int blob64, blob32;             // the chunk's blob offset in 16-byte units (FP64 / FP32 blobs)
};

// The shared-memory footprint of the sweep: the value table, then S slots of
// [blob | b | gather sources]. The sources (int positions) keep a 16-byte cover's lead.
template <class T>
__host__ __device__ inline unsigned tableBytes(int G)
{
    return r16(static_cast<unsigned>(sizeof(T)) * (kWin + kStages * G + 1));
}
template <class T>
__host__ __device__ inline unsigned slotBOffset(int M, int E, int items = 0)
{
    return blobLayout<T>(M, E, items).bytes;
}
template <class T>
__host__ __device__ inline unsigned slotListOffset(int M, int E, int items = 0)
{
    return slotBOffset<T>(M, E, items) + r16(static_cast<unsigned>(sizeof(T)) * (M + 8));
}
template <class T>
__host__ __device__ inline unsigned slotBytes(int M, int E, int G, int items = 0)
{
    return slotListOffset<T>(M, E, items) + r16(4u * (G + 8));
}
template <class T>
__host__ __device__ inline size_t gsSmemBytes(int M, int E, int G, int items = 0)
{
    return static_cast<size_t>(tableBytes<T>(G)) + kStages * static_cast<size_t>(slotBytes<T>(M, E, G, items));
}

template <class T>
struct GsArgs
{
    int nParts;
    int maxCells;                  // M: chunk cell capacity (compute threads, a multiple of 32)
    int maxEnt;                    // E: chunk ELL entry capacity (a multiple of 32)
    int maxGat;                    // G: gathered values per chunk (per stage in the table)
    int ahead;                     // window extent ahead of a chunk's start (positions)
    int nPadded;                   // psi is readable up to here (whole fill blocks)
    const int* __restrict__ partChunkStart;  // [P+1]
    const int* __restrict__ partPosStart;    // [P+1]
    const int4* __restrict__ chunkRec;       // [nChunks][3]
    const int* __restrict__ upStart;         // [P+1]
    const int* __restrict__ upList;
    const int* __restrict__ hasDown;         // [P] 1 if another part reads this part's values
    const unsigned char* __restrict__ blob;  // the chunks' blobs for this T
    const int* __restrict__ gatSrc;          // [gathers] position of each gathered value
    const T* __restrict__ b;                 // [n (+pad)] by position
    T* psi;                                  // [n] by position, updated in place (padded)
    unsigned* progress;                      // [P][kProgressStride] (word 0 of each line used)
    int* ticket;                             // the launch's part ticket (zeroed before it), or null:
                                             // part = blockIdx.x
    int items;                               // 0: one sweep, positions; 1: an item schedule (several
                                             // sweeps pipelined: "positions" index (sweep, cell)
                                             // items, b is by item, the window is not filled ahead,
                                             // and each item writes psi at its blob's storage position)
    long long spinLimit;                     // polls before a wait gives up (kSpinLimit)
    int publish;                             // 1; 0 only to test the bounded waits: no part releases
                                             // its progress, so a part that needs another's values
                                             // waits for a word nothing sets and gives up
    int* err;
    unsigned long long* trace;               // diagnostic, or null (SM clock64 stamps): [nChunks][4]
                                             // compute thread 0 (chunk start, past the depth
                                             // barrier, data ready, computed); [P][4] {globaltimer,
                                             // clock64} at the part's start and end; [nChunks][4]
                                             // staging (TMA warp start, bulk copies issued, gather
                                             // warp past its waits, gathers issued); [P][traceDepths]
                                             // [2] per depth d: when the publisher released d and
                                             // when the watcher first saw the upstream parts at d
    int traceDepths;
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
// 1-D TMA bulk copy global -> shared (32-bit shared address), completing on `bar`. dst, src
// 16-byte aligned; bytes % 16 == 0.
__device__ __forceinline__ void tmaLoad(unsigned dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     dst),
                 "l"(src), "r"(bytes), "r"(smemAddr(bar))
                 : "memory");
}
// one 8- or 4-byte cp.async global -> shared (32-bit shared address)
__device__ __forceinline__ void cpAsync(unsigned dst, const double* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cpAsync(unsigned dst, const float* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void fenceProxyAsyncShared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
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

__device__ __forceinline__ ChunkRec loadChunkRec(const int4* __restrict__ recs, int c)
{
    const int4 a = recs[3 * (size_t)c];
    const int4 b = recs[3 * (size_t)c + 1];
    const int4 d = recs[3 * (size_t)c + 2];
    ChunkRec r;
    r.pos0 = a.x; r.m = a.y; r.ent0 = a.z; r.nEnt = a.w;
    r.gat0 = b.x; r.nGat = b.y; r.depth = b.z; r.needUp = b.w;
    r.sameWait = d.x; r.newDepth = d.y & 1; r.nOld = d.y >> 1; r.blob64 = d.z; r.blob32 = d.w;
    return r;
}
template <class T>
__host__ __device__ __forceinline__ int blobOf(const ChunkRec& r)
{
    return sizeof(T) == 8 ? r.blob64 : r.blob32;
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

// Bounded waits: on running out, set the error word; once it is set, give up soon. The error word
// is one L2 line that every waiting warp of every part would read, so it is read only every few
// thousand polls: giving up a little later after another wait ran out costs nothing, a hot line
// shared by all SMs slows every hand-off.
constexpr long long kErrPollMask = 4095;
__device__ __forceinline__ bool errSet(const int* err) { return *reinterpret_cast<const volatile int*>(err) != 0; }

__device__ __forceinline__ void waitMbar(unsigned long long* b, unsigned parity, int* err, long long limit)
{
    long long it = 0;
    while (!mbarTryWait(b, parity))
    {
        if ((++it & kErrPollMask) == 0 && errSet(err)) return;
        if (it > limit)
        {
            atomicExch(err, 1);
            return;
        }
    }
}

// wait until the shared word *w >= target
__device__ __forceinline__ void waitShared(const unsigned* w, unsigned target, int* err, long long limit)
{
    long long it = 0;
    while (ldAcquireCta(w) < target)
    {
        if ((++it & kErrPollMask) == 0 && errSet(err)) return;
        if (it > limit)
        {
            atomicExch(err, 1);
            return;
        }
        __nanosleep(32);
    }
}

// K entries of a row, straight-line: the codes and coefficients (independent loads at fixed
// offsets), then the values, then the reference's rounding chain in entry order.
template <class T, int K>
__device__ __forceinline__ T rowTerms(T acc, unsigned cA, unsigned vA, unsigned tableA)
{
    unsigned c[K];
    T w[K], v[K];
#pragma unroll
    for (int q = 0; q < K; ++q)
    {
        c[q] = ldsU16(cA + 64u * q);
        w[q] = ldsT(vA + 32u * static_cast<unsigned>(sizeof(T)) * q, T());
    }
#pragma unroll
    for (int q = 0; q < K; ++q) v[q] = ldsT(tableA + static_cast<unsigned>(sizeof(T)) * c[q], T());
#pragma unroll
    for (int q = 0; q < K; ++q) acc = subRn(acc, mulRn(w[q], v[q]));
    return acc;
}

// Part p of one Gauss-Seidel sweep of one level, in position order. blockDim >= M + 128: M compute
// threads, then the TMA warp, the gather warp, the publisher warp and the watcher warp; warps
// beyond those (a batched launch sized for a larger M) leave after the set-up barrier.
template <class T>
__device__ __forceinline__ void gsSweepPart(const GsArgs<T>& a, const int p)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) unsigned long long full[kStages];
    __shared__ __align__(8) unsigned long long empty[kStages];
    __shared__ __align__(8) unsigned long long lists[kStages];  // a stage's record and gather sources
    __shared__ __align__(16) int4 srec[kStages][3];              // the staged chunk's record
    __shared__ unsigned pubDepth;     // every cell of this part below this depth is done (compute ->
                                      // publisher warp; 0x7fffffff at the end)
    __shared__ unsigned upMin;        // least progress seen among the upstream parts
    constexpr unsigned kT = sizeof(T);
    const int M = a.maxCells;
    const int G = a.maxGat;
    const unsigned tableA = smemAddr(smem);
    const unsigned slotsA = tableA + tableBytes<T>(G);
    const unsigned sb = slotBytes<T>(M, a.maxEnt, G, a.items);
    const unsigned bOff = slotBOffset<T>(M, a.maxEnt, a.items);     // b follows the blob in a slot
    const unsigned lOff = slotListOffset<T>(M, a.maxEnt, a.items);  // then the gather sources
    const int t = threadIdx.x;
    const int c0 = a.partChunkStart[p];
    const int nCh = a.partChunkStart[p + 1] - c0;
    const int nComputeWarps = M >> 5;
    // per-depth hand-off stamps of this part (diagnostic)
    unsigned long long* depthTrace =
        a.trace ? a.trace + 8 * (size_t)a.partChunkStart[a.nParts] + 4 * (size_t)a.nParts +
                      2 * (size_t)a.traceDepths * p
                : nullptr;
    if (t == 0)
    {
        stsT(tableA + kT * static_cast<unsigned>(kWin + kStages * G), T(0));  // what padding entries read
        pubDepth = nCh > 0 ? static_cast<unsigned>(a.chunkRec[3 * (size_t)c0 + 1].z) : 0x7fffffffu;
        upMin = 0u;
        for (int s = 0; s < kStages; ++s)
        {
            mbarInit(&full[s], 1 + 32);        // the TMA warp's expect_tx + the gather warp's 32 lanes
            mbarInit(&empty[s], nComputeWarps);
            mbarInit(&lists[s], 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fenceProxyAsyncShared();
    }
    __syncthreads();
    if (t >= M + 128) return;

    if (t >= M + 96)
    {
        // ---------------- watcher warp: upstream progress in ----------------
        // Polls the upstream parts' progress words back to back (relaxed loads: one L2 round trip
        // each) and publishes their least value in shared memory, with an acquire fence first, so
        // that the gathers issued on it read what the upstream parts released.
        const int lane = t - M - 96;
        const int upBeg = a.upStart[p];
        const int nUp = a.upStart[p + 1] - upBeg;
        if (nUp == 0) return;
        const int myUp = lane < nUp ? a.upList[upBeg + lane] : -1;  // parts beyond 32: read per poll
        unsigned seen = 0u;
        long long it = 0;
        while (true)
        {
            unsigned m = myUp >= 0 ? ldRelaxedGpu(&a.progress[kProgressStride * myUp]) : 0xffffffffu;
            for (int i = upBeg + 32 + lane; i < upBeg + nUp; i += 32) m = min(m, ldRelaxedGpu(&a.progress[kProgressStride * a.upList[i]]));
            for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (m > seen)
            {
                fenceAcqRelGpu();
                if (lane == 0) stReleaseCta(&upMin, m);
                if (depthTrace && lane == 0)
                {
                    const unsigned long long now = clockStamp();
                    for (unsigned d = seen + 1; d <= m && d < static_cast<unsigned>(a.traceDepths); ++d)
                        depthTrace[2 * d + 1] = now;
                }
                seen = m;
            }
            // done when every upstream part is, or when this part is (it needs no more values)
            if (seen == 0x7fffffffu || __shfl_sync(0xffffffffu, ldAcquireCta(&pubDepth), 0) == 0x7fffffffu) break;
            if ((++it & kErrPollMask) == 0)
            {
                if (__shfl_sync(0xffffffffu, errSet(a.err) ? 1 : 0, 0)) break;
                if (it > 16 * a.spinLimit)
                {
                    if (lane == 0) atomicExch(a.err, 1);
                    break;
                }
            }
        }
        return;
    }

    if (t >= M + 64)
    {
        // ---------------- publisher warp: this part's progress out ----------------
        // One lane spins on the shared pubDepth and releases each new value at GPU scope at once:
        // the release is cumulative over the psi stores the compute warps made before their barrier
        // and their release of pubDepth, which this lane acquired.
        if (t != M + 64 || a.hasDown[p] == 0 || !a.publish) return;
        unsigned published = 0xffffffffu;
        long long it = 0;
        while (true)
        {
            const unsigned v = ldAcquireCta(&pubDepth);
            if (v != published)
            {
                stRelease(&a.progress[kProgressStride * p], v);
                if (depthTrace && v < static_cast<unsigned>(a.traceDepths)) depthTrace[2 * v] = clockStamp();
                published = v;
            }
            if (v == 0x7fffffffu) break;
            if ((++it & kErrPollMask) == 0)
            {
                if (errSet(a.err)) break;
                if (it > 16 * a.spinLimit)
                {
                    atomicExch(a.err, 1);
                    break;
                }
            }
        }
        return;
    }

    if (t >= M)
    {
        // ---------------- staging: chunk j into slot j % S, by two warps ----------------
        // The TMA warp (one lane) issues the bulk copies; the gather warp issues the gathers and
        // waits for what they need, so a wait for an upstream part never delays the bulk copies of
        // the chunks behind it. Chunk records and gather sources are loaded two chunks ahead: no
        // iteration waits for a load it issued itself.
        unsigned long long* ptr = a.trace ? a.trace + 4 * (size_t)a.partChunkStart[a.nParts] + 4 * (size_t)a.nParts : nullptr;
        if (t < M + 32)
        {
            if (t != M) return;
            const int partEnd = a.partPosStart[p + 1];
            const int fillEnd = min(a.nPadded, ((partEnd + kFill - 1) / kFill) * kFill);
            int filled = (a.partPosStart[p] / kFill) * kFill;  // window filled up to here
            ChunkRec r1 = nCh > 0 ? loadChunkRec(a.chunkRec, c0) : ChunkRec{};
            ChunkRec r2 = nCh > 1 ? loadChunkRec(a.chunkRec, c0 + 1) : ChunkRec{};
            int s = 0;
            for (int j = 0; j < nCh; ++j)
            {
                const ChunkRec cr = r1;
                r1 = r2;
                if (j + 2 < nCh) r2 = loadChunkRec(a.chunkRec, c0 + j + 2);
                if (ptr) ptr[4 * (size_t)(c0 + j)] = clockStamp();
                if (j >= kStages) waitMbar(&empty[s], static_cast<unsigned>((j / kStages - 1) & 1), a.err, a.spinLimit);
                const unsigned slotA = slotsA + static_cast<unsigned>(s) * sb;
                // the record and the gather sources first: the gather warp starts from them
                const int4* rg = a.chunkRec + 3 * (size_t)(c0 + j);
                srec[s][0] = rg[0];
                srec[s][1] = rg[1];
                srec[s][2] = rg[2];
                const Cover cl = coverOf(a.gatSrc, cr.gat0, cr.nGat);
                mbarExpectTx(&lists[s], cr.nGat ? cl.bytes : 0u);
                if (cr.nGat) tmaLoad(slotA + lOff, cl.src, cl.bytes, &lists[s]);
                const BlobLayout bl = blobLayout<T>(cr.m, cr.nEnt, a.items);
                const Cover cbv = coverOf(a.b, cr.pos0, cr.m);
                // the window ahead of the front holds old psi values; an item schedule's window holds
                // item results only (its old values are gathered)
                const int target = a.items ? filled : min(fillEnd, ((cr.pos0 + a.ahead + kFill - 1) / kFill) * kFill);
                const int nFill = target > filled ? (target - filled) / kFill : 0;
                mbarExpectTx(&full[s], bl.bytes + cbv.bytes + static_cast<unsigned>(nFill) * kFill * kT);
                tmaLoad(slotA, a.blob + 16 * static_cast<size_t>(blobOf<T>(cr)), bl.bytes, &full[s]);
                tmaLoad(slotA + bOff, cbv.src, cbv.bytes, &full[s]);
                for (int f = 0; f < nFill; ++f, filled += kFill)
                    tmaLoad(tableA + kT * static_cast<unsigned>(filled & (kWin - 1)), a.psi + filled, kFill * kT,
                            &full[s]);
                if (ptr) ptr[4 * (size_t)(c0 + j) + 1] = clockStamp();
                if (++s == kStages) s = 0;
            }
            // before the CTA can exit, the last stages' copies have landed: on an error path the
            // compute warps may give up waiting for them, and no bulk copy may still be writing into
            // the shared memory of a CTA that has exited (a bulk copy always completes, so this
            // wait ends; it is bounded all the same, and not cut short by the error word)
            for (int j = max(0, nCh - kStages); j < nCh; ++j)
            {
                long long it = 0;
                while (!mbarTryWait(&full[j % kStages], static_cast<unsigned>((j / kStages) & 1)) &&
                       ++it <= a.spinLimit)
                {
                }
            }
            return;
        }
        const int lane = t - M - 32;
        int s = 0;
        unsigned phase = 0u;
        for (int j = 0; j < nCh; ++j)
        {
            // the TMA warp published this stage's record and sources once the slot was free
            waitMbar(&lists[s], phase, a.err, a.spinLimit);
            const int4 rb1 = srec[s][1];
            const int4 rb2 = srec[s][2];
            const int gat0 = rb1.x, nGat = rb1.y, needUp = rb1.w, sameWait = rb2.x, nOld = rb2.y >> 1;
            const unsigned listA = slotsA + static_cast<unsigned>(s) * sb + lOff +
                                   4u * static_cast<unsigned>(coverOf(a.gatSrc, gat0, 0).lead);
            const unsigned gA = tableA + kT * static_cast<unsigned>(kWin + s * G);
            // the old values first: they are final as they are
            for (int g = lane; g < nOld; g += 32)
                cpAsync(gA + kT * static_cast<unsigned>(g), &a.psi[static_cast<int>(ldsU32(listA + 4u * g))]);
            if (lane == 0)
            {
                // gathered new values must be final: owners of other parts once those parts are far
                // enough along, owners of this part once their chunk is consumed (chunk sw is done
                // when empty[sw % S] completes phase sw / S; the slot wait for chunk j already
                // covers every chunk up to j - S, and phase sw / S + 1 needs chunk sw + S > j, so
                // the parity is unambiguous)
                if (needUp >= 0) waitShared(&upMin, static_cast<unsigned>(needUp) + 1u, a.err, a.spinLimit);
                const int sw = sameWait - c0;
                if (sameWait >= 0 && sw > j - kStages)
                    waitMbar(&empty[sw % kStages], static_cast<unsigned>((sw / kStages) & 1), a.err, a.spinLimit);
                if (ptr) ptr[4 * (size_t)(c0 + j) + 2] = clockStamp();
            }
            __syncwarp();
            for (int g = nOld + lane; g < nGat; g += 32)
                cpAsync(gA + kT * static_cast<unsigned>(g), &a.psi[static_cast<int>(ldsU32(listA + 4u * g))]);
            mbarArriveCpAsync(&full[s]);
            if (ptr && lane == 0) ptr[4 * (size_t)(c0 + j) + 3] = clockStamp();
            if (++s == kStages)
            {
                s = 0;
                phase ^= 1u;
            }
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
    int s = 0;
    unsigned phase = 0u;
    for (int j = 0; j < nCh; ++j)
    {
        if (a.trace && t == 0) a.trace[4 * (size_t)(c0 + j)] = clockStamp();
        // the record is published with the stage's gather sources, well before the data: the
        // progress this part publishes at a depth change must not wait for this chunk's data
        waitMbar(&lists[s], phase, a.err, a.spinLimit);
        const ChunkRec cr = loadChunkRec(srec[s], 0);
        if (cr.newDepth && j > 0)
        {
            // the owners this chunk reads were computed by any compute warp: wait for all of them;
            // then every cell of this part below this chunk's depth is done
            computeSync(M);
            if (t == 0) stReleaseCta(&pubDepth, static_cast<unsigned>(cr.depth));
        }
        if (a.trace && t == 0) a.trace[4 * (size_t)(c0 + j) + 1] = clockStamp();
        waitMbar(&full[s], phase, a.err, a.spinLimit);
        if (a.trace && t == 0) a.trace[4 * (size_t)(c0 + j) + 2] = clockStamp();
        if (t < cr.m)
        {
            const unsigned slotA = slotsA + static_cast<unsigned>(s) * sb;
            const BlobLayout bl = blobLayout<T>(cr.m, cr.nEnt, a.items);
            const unsigned lb = (static_cast<unsigned>(cr.pos0) * kT & 15u) / kT;  // lead of b's cover
            const unsigned pe = ldsU32(slotA + bl.desc + 4u * t);
            T acc = ldsT(slotA + bOff + kT * (lb + t), T());
            const T dg = ldsT(slotA + kT * t, T());
            const int width = static_cast<int>(pe >> 24);
            const unsigned rb = pe & 0xffffffu;
            unsigned cA = slotA + bl.code + 2u * rb;
            unsigned vA = slotA + bl.val + kT * rb;
            int left = width;
            for (; left >= 8; left -= 8, cA += 64u * 8, vA += 32u * kT * 8) acc = rowTerms<T, 8>(acc, cA, vA, tableA);
            // the width is the same for the whole warp: this switch does not diverge
            switch (left)
            {
            case 7: acc = rowTerms<T, 7>(acc, cA, vA, tableA); break;
            case 6: acc = rowTerms<T, 6>(acc, cA, vA, tableA); break;
            case 5: acc = rowTerms<T, 5>(acc, cA, vA, tableA); break;
            case 4: acc = rowTerms<T, 4>(acc, cA, vA, tableA); break;
            case 3: acc = rowTerms<T, 3>(acc, cA, vA, tableA); break;
            case 2: acc = rowTerms<T, 2>(acc, cA, vA, tableA); break;
            case 1: acc = rowTerms<T, 1>(acc, cA, vA, tableA); break;
            default: break;
            }
            const T res = divRn(acc, dg);
            const int pos = cr.pos0 + t;
            stsT(tableA + kT * static_cast<unsigned>(pos & (kWin - 1)), res);
            // this window slot is refilled by TMA (the async proxy) one window later; the fence comes
            // before the global store so that it does not wait for that store
            fenceProxyAsyncShared();
            a.psi[a.items ? static_cast<int>(ldsU32(slotA + bl.store + 4u * t)) : pos] = res;
        }
        if (a.trace && t == 0) a.trace[4 * (size_t)(c0 + j) + 3] = clockStamp();
        __syncwarp();
        if (lane == 0) mbarArrive(&empty[s]);
        if (++s == kStages)
        {
            s = 0;
            phase ^= 1u;
        }
    }
    computeSync(M);
    if (t == 0) stReleaseCta(&pubDepth, 0x7fffffffu);
    if (ptrace && t == 0)
    {
        ptrace[2] = globalTimer();
        ptrace[3] = clockStamp();
    }
}

// FORWARD PROGRESS. A part waits only for lower-numbered parts (of its own case in a batch). A CTA
// takes its part from a ticket counter when it starts, not from blockIdx: the ticket it draws is
// held only by a CTA that is already running, so every lower-numbered part is running or done
// whatever order the hardware dispatches the blocks in, and however many other kernels share the
// SMs (several server slots, say) -- every wait is for a part that is running.
__device__ __forceinline__ int drawTicket(int* ticket)
{
    __shared__ int part;
    if (threadIdx.x == 0) part = ticket ? atomicAdd(ticket, 1) : static_cast<int>(blockIdx.x);
    __syncthreads();
    return part;
}

// One sweep of one level: grid = the level's P parts.
template <class T>
__global__ void __launch_bounds__(kMaxCompute + 128, 1) gsSweep(GsArgs<T> a)
{
    gsSweepPart<T>(a, drawTicket(a.ticket));
}

// One sweep of one level of many independent cases in ONE launch: the CTA with ticket i runs part
// parts[i].y of the case whose arguments are cases[parts[i].x]; parts[i].z indexes `active` (may be
// null), and a case whose flag is 0 is skipped. A case's parts follow each other in ticket order, and
// a part waits only for lower-numbered parts of its own case, which hold lower tickets.
template <class T>
__global__ void __launch_bounds__(kMaxCompute + 128, 1) gsSweepBatch(const GsArgs<T>* __restrict__ cases,
                                                                     const int4* __restrict__ parts,
                                                                     const int* __restrict__ active,
                                                                     int* __restrict__ ticket)
{
    __shared__ __align__(16) GsArgs<T> sa;
    const int4 cp = parts[drawTicket(ticket)];
    if (active && active[cp.z] == 0) return;
    static_assert(sizeof(GsArgs<T>) % 4 == 0, "GsArgs copied word by word");
    constexpr int kWords = static_cast<int>(sizeof(GsArgs<T>) / 4);
    const int* src = reinterpret_cast<const int*>(cases + cp.x);
    for (int i = threadIdx.x; i < kWords; i += blockDim.x) reinterpret_cast<int*>(&sa)[i] = src[i];
    __syncthreads();
    gsSweepPart<T>(sa, cp.y);
}

// The chunk blobs of one level in value type T (one block per chunk): the diagonal and row
// descriptors by position, the coefficients and codes by ELL entry.
template <class T>
__global__ void buildChunkBlobs(int nCh, const int4* __restrict__ recs, const T* __restrict__ posDiag,
                                const unsigned* __restrict__ posEnt, const unsigned short* __restrict__ code,
                                const int* __restrict__ entFace, const double* __restrict__ upper,
                                unsigned char* __restrict__ blob, const int* __restrict__ itemStore)
{
    for (int c = blockIdx.x; c < nCh; c += gridDim.x)
    {
        const ChunkRec r = loadChunkRec(recs, c);
        const BlobLayout L = blobLayout<T>(r.m, r.nEnt, itemStore ? 1 : 0);
        unsigned char* b = blob + 16 * static_cast<size_t>(blobOf<T>(r));
        T* dg = reinterpret_cast<T*>(b);
        unsigned* ds = reinterpret_cast<unsigned*>(b + L.desc);
        unsigned* st = reinterpret_cast<unsigned*>(b + L.store);
        T* vl = reinterpret_cast<T*>(b + L.val);
        unsigned short* cd = reinterpret_cast<unsigned short*>(b + L.code);
        for (int i = threadIdx.x; i < r.m; i += blockDim.x)
        {
            const int p = itemStore ? itemStore[r.pos0 + i] : r.pos0 + i;
            dg[i] = posDiag[p];
            ds[i] = posEnt[r.pos0 + i];
            if (itemStore) st[i] = static_cast<unsigned>(p);
        }
        for (int e = threadIdx.x; e < r.nEnt; e += blockDim.x)
        {
            const int f = entFace[r.ent0 + e];
            vl[e] = f >= 0 ? static_cast<T>(upper[f]) : T(0);
            cd[e] = code[r.ent0 + e];
        }
    }
}

}  // namespace k
}  // namespace b2g
