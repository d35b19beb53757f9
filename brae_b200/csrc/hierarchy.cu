// hierarchy.cu -- the faceAreaPair GAMG hierarchy, built on the device, bit-for-bit the reference's.
//
// Reference (paths relative to its project root):
//   AGG = src/matrices/lduMatrix/solvers/GAMG/GAMGAgglomerations/pair_gamg_agglomeration_cpp.cu
//
// THE PAIRING IS A SEQUENTIAL GREEDY (AGG:158-284) and is reproduced exactly by a dependency-
// counted frontier: when a cell is visited, its decision depends only on which of its neighbours
// are still unmatched, and a neighbour n is unmatched at c's visit iff n is visited after c and no
// cell visited before c has paired with n. So c can decide as soon as every cell m visited before
// it that is either c's neighbour, or the neighbour of one of c's later-visited neighbours, has
// decided. Each cell counts those (m, path) pairs; a decided cell decrements the counters of the
// cells that count it, and a counter reaching zero puts the cell on the next frontier. Within one
// frontier no two cells can touch the same later neighbour (one would count the other), so a
// frontier decides without races, and every cell decides exactly what the sequential pass decides.
// The coarse numbering (order of pair creation in visit order, singletons after, the backward
// renumbering c -> n-1-c) is then a prefix sum over visit order.
#include "hierarchy.cuh"
#include "gs_kernels.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

namespace b2g {

namespace {

constexpr int TPB = 256;
constexpr double kGreatAgg = 1.0e+15;  // scalar.H GREAT (AGG:15)
constexpr int kMaxLevels = 50;          // GAMGAgglomeration.C:248 (AGG:13)

inline int grid(long long n) { return std::max(1, ceilDiv(n, TPB)); }

int bitsFor(long long maxValue)
{
    int b = 1;
    while (b < 63 && (1LL << b) <= maxValue) ++b;
    return b;
}

// ---------------------------------------------------------------------------------------------
// layouts
// ---------------------------------------------------------------------------------------------

__global__ void kCheckOrder(int nF, int nC, const int* __restrict__ lower, const int* __restrict__ upper,
                            int* err)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    const int l = lower[f];
    const int u = upper[f];
    if (l < 0 || u < 0 || l >= nC || u >= nC) { atomicOr(err, 1); return; }
    if (l >= u) atomicOr(err, 2);
    if (f > 0 && l < lower[f - 1]) atomicOr(err, 4);
}

__global__ void kCount(const int* __restrict__ keys, int n, int* counts)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(&counts[keys[i]], 1);
}

__global__ void kIota(int* v, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

__global__ void kAddInts(const int* a, const int* b, int* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[i] + b[i];
}

__global__ void kFillRows(int nC, const int* __restrict__ lower, const int* __restrict__ upper,
                          const int* __restrict__ ownStart, const int* __restrict__ losortStart,
                          const int* __restrict__ losort, const int* __restrict__ rowStart,
                          int* __restrict__ col, int* __restrict__ entFace)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    int k = rowStart[c];
    for (int q = losortStart[c]; q < losortStart[c + 1]; ++q)
    {
        const int f = losort[q];
        col[k] = lower[f];
        entFace[k] = f;
        ++k;
    }
    for (int f = ownStart[c]; f < ownStart[c + 1]; ++f)
    {
        col[k] = upper[f];
        entFace[k] = f;
        ++k;
    }
}

// ---------------------------------------------------------------------------------------------
// pairing (AGG:158-284)
// ---------------------------------------------------------------------------------------------

enum : int { ST_UNDECIDED = 0, ST_CREATOR = 1, ST_TAKEN = 2, ST_JOINER = 3, ST_LONE = 4 };

__device__ __forceinline__ int rankOf(int c, int n, int fwd) { return fwd ? c : n - 1 - c; }

// mag(cmptMultiply(Sf/sqrt(magSf), (1, 1.01, 1.02))) (AGG:301-311), every operation rounded
__global__ void kFaceWeights(int nF, const double* __restrict__ Sf, const double* __restrict__ magSf,
                             double* __restrict__ w)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    const double r = __dsqrt_rn(magSf[f]);
    const double wx = __ddiv_rn(Sf[3 * (size_t)f], r);
    const double wy = __dmul_rn(__ddiv_rn(Sf[3 * (size_t)f + 1], r), 1.01);
    const double wz = __dmul_rn(__ddiv_rn(Sf[3 * (size_t)f + 2], r), 1.02);
    w[f] = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(wx, wx), __dmul_rn(wy, wy)), __dmul_rn(wz, wz)));
}

// c counts every (m, path) it must wait for: its earlier neighbours, and for each later neighbour
// n, n's neighbours visited before c.
__global__ void kPairCounters(int n, int fwd, const int* __restrict__ rowStart, const int* __restrict__ col,
                              int* __restrict__ ctr)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int r = rankOf(c, n, fwd);
    int k = 0;
    for (int e = rowStart[c]; e < rowStart[c + 1]; ++e)
    {
        const int m = col[e];
        const int rm = rankOf(m, n, fwd);
        if (rm < r)
        {
            ++k;
        }
        else if (rm > r)
        {
            for (int e2 = rowStart[m]; e2 < rowStart[m + 1]; ++e2)
            {
                if (rankOf(col[e2], n, fwd) < r) ++k;
            }
        }
    }
    ctr[c] = k;
}

__global__ void kSeedFrontier(int n, const int* __restrict__ ctr, int* __restrict__ frontier, int* size)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n && ctr[c] == 0) frontier[atomicAdd(size, 1)] = c;
}

__global__ void kPairRound(int n, int fwd, const int* __restrict__ frontier, int fsize,
                           const int* __restrict__ rowStart, const int* __restrict__ col,
                           const int* __restrict__ entFace, const double* __restrict__ w,
                           int* __restrict__ st, int* __restrict__ partner, int* __restrict__ target,
                           int* __restrict__ ctr, int* __restrict__ next, int* nextSize)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= fsize) return;
    const int c = frontier[t];
    const int r = rankOf(c, n, fwd);
    const int rb = rowStart[c];
    const int re = rowStart[c + 1];
    if (st[c] != ST_TAKEN)
    {
        // the first face of maximum weight, in cellFaces order, whose other cell is unmatched
        int best = -1;
        double bestW = -kGreatAgg;
        for (int e = rb; e < re; ++e)
        {
            const int nb = col[e];
            const bool avail = rankOf(nb, n, fwd) > r && st[nb] != ST_TAKEN;
            const double we = w[entFace[e]];
            if (avail && we > bestW)
            {
                best = e;
                bestW = we;
            }
        }
        if (best >= 0)
        {
            const int nb = col[best];
            partner[c] = nb;
            partner[nb] = c;
            st[nb] = ST_TAKEN;
            st[c] = ST_CREATOR;
        }
        else
        {
            // no unmatched neighbour: join the cluster across the heaviest face (AGG:239-257)
            int cbest = -1;
            double cw = -kGreatAgg;
            for (int e = rb; e < re; ++e)
            {
                const double we = w[entFace[e]];
                if (we > cw)
                {
                    cbest = e;
                    cw = we;
                }
            }
            if (cbest >= 0)
            {
                target[c] = col[cbest];
                st[c] = ST_JOINER;
            }
            else
            {
                st[c] = ST_LONE;
            }
        }
    }
    // release the cells that counted c
    for (int e = rb; e < re; ++e)
    {
        const int m = col[e];
        const int rm = rankOf(m, n, fwd);
        if (rm > r)
        {
            if (atomicSub(&ctr[m], 1) == 1) next[atomicAdd(nextSize, 1)] = m;
        }
        for (int e2 = rowStart[m]; e2 < rowStart[m + 1]; ++e2)
        {
            const int d = col[e2];
            const int rd = rankOf(d, n, fwd);
            if (rd > r && rd < rm)
            {
                if (atomicSub(&ctr[d], 1) == 1) next[atomicAdd(nextSize, 1)] = d;
            }
        }
    }
}

// rank-ordered flags: creators (for pair numbering) and lone cells (singletons)
__global__ void kRankFlags(int n, int fwd, const int* __restrict__ st, int* __restrict__ isCreator,
                           int* __restrict__ isLone)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int c = fwd ? r : n - 1 - r;
    isCreator[r] = st[c] == ST_CREATOR;
    isLone[r] = st[c] == ST_LONE || st[c] == ST_UNDECIDED;
}

__global__ void kAssignPairs(int n, int fwd, const int* __restrict__ st, const int* __restrict__ partner,
                             const int* __restrict__ creatorId, const int* __restrict__ loneId, int nPairs,
                             int* __restrict__ map)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int r = rankOf(c, n, fwd);
    const int s = st[c];
    if (s == ST_CREATOR) map[c] = creatorId[r];
    else if (s == ST_TAKEN) map[c] = creatorId[rankOf(partner[c], n, fwd)];
    else if (s == ST_LONE || s == ST_UNDECIDED) map[c] = nPairs + loneId[r];
}

__global__ void kAssignJoiners(int n, const int* __restrict__ st, const int* __restrict__ target,
                               int* __restrict__ map)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n || st[c] != ST_JOINER) return;
    int t = target[c];
    for (int guard = 0; st[t] == ST_JOINER && guard < n; ++guard) t = target[t];
    map[c] = map[t];
}

__global__ void kReverseMap(int n, int nCoarse, int* map)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) map[c] = (nCoarse - 1) - map[c];
}

// ---------------------------------------------------------------------------------------------
// coarse addressing (AGG:28-154) and weight restriction (AGG:328-339)
// ---------------------------------------------------------------------------------------------

__global__ void kFaceKeys(int nF, const int* __restrict__ lower, const int* __restrict__ upper,
                          const int* __restrict__ map, unsigned long long internalKey,
                          unsigned long long* __restrict__ keys, int* __restrict__ fr, int* nInternal)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    const int ru = map[upper[f]];
    const int rl = map[lower[f]];
    if (ru == rl)
    {
        fr[f] = -(ru + 1);
        keys[f] = internalKey;
        atomicAdd(nInternal, 1);
        return;
    }
    const unsigned long long o = static_cast<unsigned>(min(ru, rl));
    const unsigned long long nb = static_cast<unsigned>(max(ru, rl));
    keys[f] = (o << 32) | nb;
}

__global__ void kSegHeads(int nValid, const unsigned long long* __restrict__ keys, int* __restrict__ head)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nValid) return;
    head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// per unique (owner, neighbour) pair: its fine-face segment and first appearance
__global__ void kUniqueInfo(int nValid, const unsigned long long* __restrict__ keys,
                            const int* __restrict__ faces, const int* __restrict__ head,
                            const int* __restrict__ segScan, unsigned long long* __restrict__ key2,
                            int* __restrict__ uBeg)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nValid || !head[i]) return;
    const int u = segScan[i];
    const unsigned long long own = keys[i] >> 32;
    key2[u] = (own << 32) | static_cast<unsigned>(faces[i]);  // owner-major, then first appearance
    uBeg[u] = i;
}

__global__ void kCoarseFaces(int nUnique, int nValid, const unsigned long long* __restrict__ sortedKeys,
                             const int* __restrict__ uOrder, const int* __restrict__ uBeg,
                             const unsigned long long* __restrict__ keys, int* __restrict__ cLower,
                             int* __restrict__ cUpper, int* __restrict__ faceBeg, int* __restrict__ faceEnd,
                             int* __restrict__ cfOfU)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nUnique) return;
    const int u = uOrder[p];
    const int b = uBeg[u];
    const unsigned long long k = keys[b];
    cLower[p] = static_cast<int>(k >> 32);
    cUpper[p] = static_cast<int>(k & 0xffffffffULL);
    faceBeg[p] = b;
    faceEnd[p] = (u + 1 < nUnique) ? uBeg[u + 1] : nValid;
    cfOfU[u] = p;
}

// segIncl is the inclusive scan of segment heads: element i belongs to unique pair segIncl[i] - 1
__global__ void kFaceRestrict(int nValid, const int* __restrict__ faces, const int* __restrict__ segIncl,
                              const int* __restrict__ cfOfU, int* __restrict__ fr)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nValid) return;
    fr[faces[i]] = cfOfU[segIncl[i] - 1];
}

__global__ void kFlip(int nF, const int* __restrict__ lower, const int* __restrict__ upper,
                      const int* __restrict__ map, const int* __restrict__ fr, int8_t* __restrict__ flip)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    // true where the fine face's UPPER cell fell in the coarse OWNER (AGG:127-148)
    flip[f] = (fr[f] >= 0 && map[upper[f]] < map[lower[f]]) ? 1 : 0;
}

// next-level weights: each coarse face sums its fine faces' weights in ascending fine face
__global__ void kRestrictWeights(int nCF, const int* __restrict__ faceBeg, const int* __restrict__ faceEnd,
                                 const int* __restrict__ faceList, const double* __restrict__ w,
                                 double* __restrict__ cw)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nCF) return;
    double s = 0.0;
    for (int i = faceBeg[p]; i < faceEnd[p]; ++i) s = __dadd_rn(s, w[faceList[i]]);
    cw[p] = s;
}

__global__ void kInternalKeys(int nInt, const int* __restrict__ faces, const int* __restrict__ fr,
                              unsigned* __restrict__ keys)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nInt) keys[i] = static_cast<unsigned>(-1 - fr[faces[i]]);
}

__global__ void kKeysToInt(int n, const unsigned* __restrict__ k, int* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = static_cast<int>(k[i]);
}

// ---------------------------------------------------------------------------------------------
// Gauss-Seidel schedule: depths (Kahn's frontier) and parts
// ---------------------------------------------------------------------------------------------

__global__ void kIndegree(int n, const int* __restrict__ losortStart, int* __restrict__ indeg,
                          int* __restrict__ frontier, int* size)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int d = losortStart[c + 1] - losortStart[c];
    indeg[c] = d;
    if (d == 0) frontier[atomicAdd(size, 1)] = c;
}

__global__ void kDepthRound(int round, const int* __restrict__ frontier, int fsize,
                            const int* __restrict__ ownStart, const int* __restrict__ upper,
                            int* __restrict__ indeg, int* __restrict__ depth, int* __restrict__ next,
                            int* nextSize)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= fsize) return;
    const int c = frontier[t];
    depth[c] = round;
    for (int f = ownStart[c]; f < ownStart[c + 1]; ++f)
    {
        const int nb = upper[f];
        if (atomicSub(&indeg[nb], 1) == 1) next[atomicAdd(nextSize, 1)] = nb;
    }
}

__global__ void kPartOf(int n, int nParts, const int* __restrict__ partStart, int* __restrict__ partOf)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    int lo = 0, hi = nParts - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (partStart[mid] <= c) lo = mid; else hi = mid - 1;
    }
    partOf[c] = lo;
}

__global__ void kSchedKeys(int n, int stride, const int* __restrict__ partOf, const int* __restrict__ depth,
                           unsigned* __restrict__ keys)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) keys[c] = static_cast<unsigned>(partOf[c]) * static_cast<unsigned>(stride) +
                         static_cast<unsigned>(depth[c]);
}

__global__ void kKeyHeads(int n, const unsigned* __restrict__ keys, int* __restrict__ head)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

__global__ void kLevelInfo(int n, int stride, const unsigned* __restrict__ keys, const int* __restrict__ head,
                           const int* __restrict__ lvlScan, int* __restrict__ lvlStart,
                           int* __restrict__ lvlDepth, int* __restrict__ lvlPart)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !head[i]) return;
    const int L = lvlScan[i];
    lvlStart[L] = i;
    lvlDepth[L] = static_cast<int>(keys[i] % static_cast<unsigned>(stride));
    lvlPart[L] = static_cast<int>(keys[i] / static_cast<unsigned>(stride));
}

// part boundaries: part p starts at the first cell whose cumulative cost (cells + row entries)
// reaches total*p/P
__global__ void kPartBounds(int n, int P, const int* __restrict__ rowStart, int* __restrict__ partStart)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > P) return;
    if (p == 0) { partStart[0] = 0; return; }
    if (p == P) { partStart[P] = n; return; }
    const long long total = static_cast<long long>(n) + rowStart[n];
    const long long target = total * p / P;
    int lo = 0, hi = n;
    while (lo < hi)
    {
        const int mid = (lo + hi) >> 1;
        if (static_cast<long long>(mid) + rowStart[mid] < target) lo = mid + 1; else hi = mid;
    }
    partStart[p] = lo;
}

__global__ void kStepCounts(int nCoarse, const int* __restrict__ posCellC, const int* __restrict__ cellStart,
                            int* __restrict__ cnt)
{
    const int P = blockIdx.x * blockDim.x + threadIdx.x;
    if (P >= nCoarse) return;
    const int C = posCellC[P];
    cnt[P] = cellStart[C + 1] - cellStart[C];
}

__global__ void kStepLists(int nCoarse, const int* __restrict__ posCellC, const int* __restrict__ cellStart,
                           const int* __restrict__ cellList, const int* __restrict__ posOfF,
                           const int* __restrict__ rStartP, int* __restrict__ rListP)
{
    const int P = blockIdx.x * blockDim.x + threadIdx.x;
    if (P >= nCoarse) return;
    const int C = posCellC[P];
    int k = rStartP[P];
    for (int e = cellStart[C]; e < cellStart[C + 1]; ++e) rListP[k++] = posOfF[cellList[e]];
}

__global__ void kProlongMap(int nFine, const int* __restrict__ posCellF, const int* __restrict__ restrictAddr,
                            const int* __restrict__ posOfC, int* __restrict__ prolongP)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nFine) prolongP[i] = posOfC[restrictAddr[posCellF[i]]];
}

__global__ void kPosOf(int n, const int* __restrict__ order, int* __restrict__ posOf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) posOf[order[i]] = i;
}

__global__ void kPosRowLen(int n, const int* __restrict__ order, const int* __restrict__ rowStart,
                           int* __restrict__ len)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) len[i] = rowStart[order[i] + 1] - rowStart[order[i]];
}

// CSR rows in position order (the Amul, residual and reduction kernels): the other cell's position
// and the face, per entry
__global__ void kCsrPositions(int n, const int* __restrict__ order, const int* __restrict__ posOf,
                              const int* __restrict__ rowStart, const int* __restrict__ col,
                              const int* __restrict__ entFace, const int* __restrict__ posRow,
                              int* __restrict__ colPos, int* __restrict__ facePos)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = order[i];
    const int base = posRow[i];
    for (int e = rowStart[c]; e < rowStart[c + 1]; ++e)
    {
        colPos[base + e - rowStart[c]] = posOf[col[e]];
        facePos[base + e - rowStart[c]] = entFace[e];
    }
}

// a 32-position slice's width, times 32: its longest row
__global__ void kEllWidth(int n, int nSlices, const int* __restrict__ posRow, int* __restrict__ width32)
{
    const int sl = blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= nSlices) return;
    int w = 0;
    for (int i = 32 * sl; i < min(n, 32 * sl + 32); ++i) w = max(w, posRow[i + 1] - posRow[i]);
    width32[sl] = 32 * w;
}

// entry q of the row in lane l of slice s at base[s] + 32*q + l; -1 past the row's end
__global__ void kEllFill(int n, const int* __restrict__ posRow, const int* __restrict__ colPos,
                         const int* __restrict__ base, int* __restrict__ ellCol, int* __restrict__ ellEnt)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int sl = static_cast<int>(t >> 5), lane = static_cast<int>(t & 31);
    if (sl * 32LL >= n) return;
    const int i = 32 * sl + lane;
    const int b0 = base[sl];
    const int w = (base[sl + 1] - b0) >> 5;
    const int r0 = i < n ? posRow[i] : 0;
    const int len = i < n ? posRow[i + 1] - r0 : 0;
    for (int q = 0; q < w; ++q)
    {
        const int e = b0 + 32 * q + lane;
        ellCol[e] = q < len ? colPos[r0 + q] : -1;
        ellEnt[e] = q < len ? r0 + q : -1;
    }
}

__global__ void kChunkOfPos(int n, int nChunks, const int* __restrict__ chunkStart, int* __restrict__ chunkOf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int lo = 0, hi = nChunks - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (chunkStart[mid] <= i) lo = mid; else hi = mid - 1;
    }
    chunkOf[i] = lo;
}

// Classification of a sweep entry (gs_kernels.cuh), for the cell at position i of chunk ch and its
// entry k (CSR row order: the faces the cell is the neighbour of, then the faces it owns). Returns
// true for a window read (slot in *code), false for a gather.
struct EntryClass
{
    int win, ahead, behind;
    const int* partOf;
    const int* chunkOf;
    const int* chunkStart;
    __device__ bool window(bool lowerSide, bool samePart, int q, int ch) const
    {
        if (!samePart) return false;
        if (lowerSide) return q >= chunkStart[ch + 1] - behind;  // an owner's new value, just behind
        return q < chunkStart[ch] + ahead;                       // a neighbour's old value, just ahead
    }
};

// pass 1: gathers per position, of old values (neighbours: final as they are) and of new values
// (owners); per chunk the waits the new ones need (other parts' owners: their deepest depth; this
// part's owners outside the window: their latest chunk), and the upstream part bits
__global__ void kGatherCounts(int n, EntryClass ec, const int* __restrict__ order, const int* __restrict__ posOf,
                              const int* __restrict__ depth, const int* __restrict__ rowStart,
                              const int* __restrict__ losortStart, const int* __restrict__ col,
                              int* __restrict__ cntOld, int* __restrict__ cntNew, int* __restrict__ chunkNeedUp,
                              int* __restrict__ chunkSameWait, unsigned* __restrict__ upBits, int words)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = order[i];
    const int p = ec.partOf[c];
    const int ch = ec.chunkOf[i];
    const int rb = rowStart[c];
    const int nLower = losortStart[c + 1] - losortStart[c];
    int gOld = 0, gNew = 0;
    for (int e = rb; e < rowStart[c + 1]; ++e)
    {
        const int o = col[e];
        const int q = posOf[o];
        const bool lowerSide = e - rb < nLower;
        const bool same = ec.partOf[o] == p;
        if (ec.window(lowerSide, same, q, ch)) continue;
        if (!lowerSide)
        {
            ++gOld;  // an old value: final as it is
            continue;
        }
        ++gNew;
        if (same)
            atomicMax(&chunkSameWait[ch], ec.chunkOf[q]);
        else
        {
            atomicMax(&chunkNeedUp[ch], depth[o]);
            const int po = ec.partOf[o];
            atomicOr(&upBits[(size_t)p * words + (po >> 5)], 1u << (po & 31));
        }
    }
    cntOld[i] = gOld;
    cntNew[i] = gNew;
}

// pass 2: the sliced-ELL entries (codes and faces) and the gather lists, each chunk's list holding
// its old values first, then its new ones; entries past a row's end keep the padding code and
// face -1 they were filled with
__global__ void kSweepEntries(int n, EntryClass ec, int maxGat, const int* __restrict__ partChunkStart,
                              const int* __restrict__ order, const int* __restrict__ posOf,
                              const int* __restrict__ rowStart, const int* __restrict__ losortStart,
                              const int* __restrict__ col, const int* __restrict__ entFace,
                              const unsigned* __restrict__ posEnt, const long long* __restrict__ chunkEnt0,
                              const int* __restrict__ oldOff, const int* __restrict__ newOff,
                              unsigned short* __restrict__ code, int* __restrict__ face, int* __restrict__ gatSrc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = order[i];
    const int p = ec.partOf[c];
    const int ch = ec.chunkOf[i];
    const int rb = rowStart[c];
    const int nLower = losortStart[c + 1] - losortStart[c];
    const long long ell = chunkEnt0[ch] + static_cast<long long>(posEnt[i] & 0xffffffu);
    // the chunk's gathered values sit in its stage's part of the value table
    const int stage = (ch - partChunkStart[p]) % k::kStages;
    const int cs = ec.chunkStart[ch];
    const int ce = ec.chunkStart[ch + 1];
    const int base = oldOff[cs] + newOff[cs];
    const int g0 = base - (k::kWin + stage * maxGat);
    int gOld = base + (oldOff[i] - oldOff[cs]);
    int gNew = base + (oldOff[ce] - oldOff[cs]) + (newOff[i] - newOff[cs]);
    for (int e = rb; e < rowStart[c + 1]; ++e)
    {
        const int k = e - rb;
        const int o = col[e];
        const int q = posOf[o];
        const bool same = ec.partOf[o] == p;
        unsigned short cd;
        if (ec.window(k < nLower, same, q, ch)) cd = static_cast<unsigned short>(q & (ec.win - 1));
        else
        {
            int& g = k < nLower ? gNew : gOld;
            cd = static_cast<unsigned short>(g - g0);
            gatSrc[g++] = q;
        }
        code[ell + 32LL * k] = cd;
        face[ell + 32LL * k] = entFace[e];
    }
}

__global__ void kChunkRecs(int nCh, const int* __restrict__ chunkStart, const long long* __restrict__ chunkEnt0,
                           const int* __restrict__ chunkDepth, const int* __restrict__ chunkNewDepth,
                           const int* __restrict__ oldOff, const int* __restrict__ newOff,
                           const int* __restrict__ chunkNeedUp,
                           const int* __restrict__ chunkSameWait, const int2* __restrict__ chunkBlob,
                           int* __restrict__ rec)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nCh) return;
    const int p0 = chunkStart[c];
    const int p1 = chunkStart[c + 1];
    int* r = rec + 12 * (size_t)c;
    r[0] = p0;
    r[1] = p1 - p0;
    r[2] = static_cast<int>(chunkEnt0[c]);
    r[3] = static_cast<int>(chunkEnt0[c + 1] - chunkEnt0[c]);
    const int nOld = oldOff[p1] - oldOff[p0];
    r[4] = oldOff[p0] + newOff[p0];
    r[5] = nOld + newOff[p1] - newOff[p0];
    r[6] = chunkDepth[c];
    r[7] = chunkNeedUp[c];
    r[8] = chunkSameWait[c];
    r[9] = chunkNewDepth[c] | (nOld << 1);
    r[10] = chunkBlob[c].x;
    r[11] = chunkBlob[c].y;
}

__global__ void kFillShort(unsigned short* v, long long n, unsigned short value)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[i] = value;
}

__global__ void kFillInt(int* v, int n, int value)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = value;
}

int readInt(const int* d, cudaStream_t s)
{
    int h = 0;
    B2G_CUDA(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, s));
    B2G_CUDA(cudaStreamSynchronize(s));
    return h;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// primitives
// ---------------------------------------------------------------------------------------------

long long exclusiveScan(const int* in, int* out, int n, cudaStream_t s)
{
    B2G_CUDA(cudaMemsetAsync(out, 0, sizeof(int), s));
    if (n == 0) return 0;
    size_t tmpBytes = 0;
    B2G_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmpBytes, in, out + 1, n, s));
    DBuf<unsigned char> tmp;
    tmp.alloc(tmpBytes, s);
    B2G_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, tmpBytes, in, out + 1, n, s));
    return readInt(out + n, s);
}

void sortPairs(const unsigned* kin, unsigned* kout, const int* vin, int* vout, int n, int bits,
               cudaStream_t s)
{
    if (n == 0) return;
    size_t tmpBytes = 0;
    B2G_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmpBytes, kin, kout, vin, vout, n, 0, bits, s));
    DBuf<unsigned char> tmp;
    tmp.alloc(tmpBytes, s);
    B2G_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmpBytes, kin, kout, vin, vout, n, 0, bits, s));
}

void sortPairs64(const unsigned long long* kin, unsigned long long* kout, const int* vin, int* vout,
                 int n, int bits, cudaStream_t s)
{
    if (n == 0) return;
    size_t tmpBytes = 0;
    B2G_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmpBytes, kin, kout, vin, vout, n, 0, bits, s));
    DBuf<unsigned char> tmp;
    tmp.alloc(tmpBytes, s);
    B2G_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmpBytes, kin, kout, vin, vout, n, 0, bits, s));
}

void countingStarts(const int* keys, int n, int nBins, int* start, cudaStream_t s)
{
    DBuf<int> counts;
    counts.alloc(static_cast<size_t>(nBins), s);
    counts.zero(s);
    if (n) kCount<<<grid(n), TPB, 0, s>>>(keys, n, counts.p);
    B2G_LAUNCH_CHECK();
    exclusiveScan(counts.p, start, nBins, s);
}

// ---------------------------------------------------------------------------------------------
// per-level layouts
// ---------------------------------------------------------------------------------------------

void buildLevelLayouts(LevelAddr& L, cudaStream_t s)
{
    const int nC = L.nCells;
    const int nF = L.nFaces;
    {
        DBuf<int> err;
        err.alloc(1, s);
        err.zero(s);
        if (nF) kCheckOrder<<<grid(nF), TPB, 0, s>>>(nF, nC, L.lower.p, L.upper.p, err.p);
        B2G_LAUNCH_CHECK();
        const int e = readInt(err.p, s);
        if (e & 1) fail(B2G_ERR_ARGUMENT, "b2g: a face's owner or neighbour is outside [0, nCells).");
        if (e & 6)
            fail(B2G_ERR_ARGUMENT,
                 "b2g: the internal faces break OpenFOAM's upper-triangular order (faces sorted by owner, "
                 "owner < neighbour). The Gauss-Seidel smoother walks the faces each cell owns through "
                 "ownerStartAddr, which only exists for a mesh ordered that way (smooth_solver_cpp.cu:10-34).");
    }
    L.ownStart.alloc(nC + 1, s);
    countingStarts(L.lower.p, nF, nC, L.ownStart.p, s);
    L.losortStart.alloc(nC + 1, s);
    countingStarts(L.upper.p, nF, nC, L.losortStart.p, s);
    // losort: faces ordered by neighbour, stable so ascending face within a cell
    L.losort.alloc(nF, s);
    {
        DBuf<int> iota;
        iota.alloc(nF, s);
        if (nF) kIota<<<grid(nF), TPB, 0, s>>>(iota.p, nF);
        DBuf<unsigned> kout;
        kout.alloc(nF, s);
        sortPairs(reinterpret_cast<const unsigned*>(L.upper.p), kout.p, iota.p, L.losort.p, nF,
                  bitsFor(nC), s);
    }
    L.rowStart.alloc(nC + 1, s);
    kAddInts<<<grid(nC + 1), TPB, 0, s>>>(L.losortStart.p, L.ownStart.p, L.rowStart.p, nC + 1);
    L.col.alloc(2 * (size_t)nF, s);
    L.entFace.alloc(2 * (size_t)nF, s);
    if (nC)
        kFillRows<<<grid(nC), TPB, 0, s>>>(nC, L.lower.p, L.upper.p, L.ownStart.p, L.losortStart.p,
                                           L.losort.p, L.rowStart.p, L.col.p, L.entFace.p);
    B2G_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------------------------
// one pairing pass: gamgPairAgglomerate (AGG:158-284)
// ---------------------------------------------------------------------------------------------

static int pairPass(const LevelAddr& L, const double* w, int fwd, DBuf<int>& map, cudaStream_t s)
{
    const int n = L.nCells;
    DBuf<int> st, partner, target, ctr, fa, fb, sizes;
    st.alloc(n, s); st.zero(s);
    partner.alloc(n, s);
    target.alloc(n, s);
    ctr.alloc(n, s);
    fa.alloc(n, s);
    fb.alloc(n, s);
    sizes.alloc(2, s);
    sizes.zero(s);
    kPairCounters<<<grid(n), TPB, 0, s>>>(n, fwd, L.rowStart.p, L.col.p, ctr.p);
    kSeedFrontier<<<grid(n), TPB, 0, s>>>(n, ctr.p, fa.p, sizes.p);
    B2G_LAUNCH_CHECK();
    int fsize = readInt(sizes.p, s);
    int* cur = fa.p;
    int* nxt = fb.p;
    int resolved = 0;
    int pinned[2];
    while (fsize > 0)
    {
        resolved += fsize;
        B2G_CUDA(cudaMemsetAsync(sizes.p + 1, 0, sizeof(int), s));
        kPairRound<<<grid(fsize), TPB, 0, s>>>(n, fwd, cur, fsize, L.rowStart.p, L.col.p, L.entFace.p, w,
                                               st.p, partner.p, target.p, ctr.p, nxt, sizes.p + 1);
        B2G_LAUNCH_CHECK();
        B2G_CUDA(cudaMemcpyAsync(pinned, sizes.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
        B2G_CUDA(cudaStreamSynchronize(s));
        fsize = pinned[1];
        B2G_CUDA(cudaMemcpyAsync(sizes.p, sizes.p + 1, sizeof(int), cudaMemcpyDeviceToDevice, s));
        std::swap(cur, nxt);
    }
    if (resolved != n)
        fail(B2G_ERR_STATE, "b2g: the agglomeration frontier stopped with " + std::to_string(n - resolved) +
                                " of " + std::to_string(n) + " cells undecided.");
    // numbering: pairs in order of creation along the visit order, then singletons
    DBuf<int> isCre, isLone, creId, loneId;
    isCre.alloc(n, s);
    isLone.alloc(n, s);
    creId.alloc(n + 1, s);
    loneId.alloc(n + 1, s);
    kRankFlags<<<grid(n), TPB, 0, s>>>(n, fwd, st.p, isCre.p, isLone.p);
    const int nPairs = static_cast<int>(exclusiveScan(isCre.p, creId.p, n, s));
    const int nLone = static_cast<int>(exclusiveScan(isLone.p, loneId.p, n, s));
    map.alloc(n, s);
    kAssignPairs<<<grid(n), TPB, 0, s>>>(n, fwd, st.p, partner.p, creId.p, loneId.p, nPairs, map.p);
    kAssignJoiners<<<grid(n), TPB, 0, s>>>(n, st.p, target.p, map.p);
    const int nCoarse = nPairs + nLone;
    if (!fwd) kReverseMap<<<grid(n), TPB, 0, s>>>(n, nCoarse, map.p);
    B2G_LAUNCH_CHECK();
    return nCoarse;
}

// ---------------------------------------------------------------------------------------------
// agglomerateLduAddressing (AGG:28-154) + restrictFaceField (AGG:328-339)
// ---------------------------------------------------------------------------------------------

static void coarseAddressing(const LevelAddr& F, Step& S, LevelAddr& Cl, const double* w,
                             DBuf<double>& cw, cudaStream_t s)
{
    const int nF = F.nFaces;
    const int nC = S.nCoarse;
    S.faceRestrict.alloc(nF, s);
    S.flip.alloc(nF, s);
    DBuf<unsigned long long> keys, skeys;
    DBuf<int> iota, faces, nInt;
    nInt.alloc(1, s);
    nInt.zero(s);
    keys.alloc(nF, s);
    skeys.alloc(nF, s);
    iota.alloc(nF, s);
    faces.alloc(nF, s);
    const int cbits = bitsFor(nC);
    const unsigned long long internalKey = (static_cast<unsigned long long>(nC) << 32);
    if (nF)
    {
        kFaceKeys<<<grid(nF), TPB, 0, s>>>(nF, F.lower.p, F.upper.p, S.restrictAddr.p, internalKey, keys.p,
                                           S.faceRestrict.p, nInt.p);
        kIota<<<grid(nF), TPB, 0, s>>>(iota.p, nF);
        B2G_LAUNCH_CHECK();
    }
    sortPairs64(keys.p, skeys.p, iota.p, faces.p, nF, 32 + cbits, s);
    // faces between two different coarse cells sort before the internal ones
    const int nValid = nF - readInt(nInt.p, s);
    DBuf<int> head, segScan, segIncl;
    head.alloc(nValid, s);
    segScan.alloc(nValid + 1, s);
    if (nValid) kSegHeads<<<grid(nValid), TPB, 0, s>>>(nValid, skeys.p, head.p);
    B2G_LAUNCH_CHECK();
    const int nUnique = static_cast<int>(exclusiveScan(head.p, segScan.p, nValid, s));
    DBuf<unsigned long long> key2, skey2;
    DBuf<int> uBeg, uIota, uOrder, cfOfU;
    key2.alloc(nUnique, s);
    skey2.alloc(nUnique, s);
    uBeg.alloc(nUnique, s);
    uIota.alloc(nUnique, s);
    uOrder.alloc(nUnique, s);
    cfOfU.alloc(nUnique, s);
    if (nValid) kUniqueInfo<<<grid(nValid), TPB, 0, s>>>(nValid, skeys.p, faces.p, head.p, segScan.p, key2.p, uBeg.p);
    if (nUnique) kIota<<<grid(nUnique), TPB, 0, s>>>(uIota.p, nUnique);
    B2G_LAUNCH_CHECK();
    sortPairs64(key2.p, skey2.p, uIota.p, uOrder.p, nUnique, 32 + cbits, s);
    Cl.nCells = nC;
    Cl.nFaces = nUnique;
    Cl.lower.alloc(nUnique, s);
    Cl.upper.alloc(nUnique, s);
    S.faceBeg.alloc(nUnique, s);
    S.faceEnd.alloc(nUnique, s);
    if (nUnique)
        kCoarseFaces<<<grid(nUnique), TPB, 0, s>>>(nUnique, nValid, skey2.p, uOrder.p, uBeg.p, skeys.p,
                                                   Cl.lower.p, Cl.upper.p, S.faceBeg.p, S.faceEnd.p, cfOfU.p);
    B2G_LAUNCH_CHECK();
    if (nValid)
    {
        // segScan[i+1] is the inclusive count of heads up to i
        kFaceRestrict<<<grid(nValid), TPB, 0, s>>>(nValid, faces.p, segScan.p + 1, cfOfU.p, S.faceRestrict.p);
        B2G_LAUNCH_CHECK();
    }
    S.nCoarseFaces = nUnique;
    if (nF) kFlip<<<grid(nF), TPB, 0, s>>>(nF, F.lower.p, F.upper.p, S.restrictAddr.p, S.faceRestrict.p, S.flip.p);
    B2G_LAUNCH_CHECK();
    // fine faces grouped by coarse face (the valid part of the sorted order)
    S.faceList.alloc(nValid, s);
    if (nValid)
        B2G_CUDA(cudaMemcpyAsync(S.faceList.p, faces.p, sizeof(int) * nValid, cudaMemcpyDeviceToDevice, s));
    cw.alloc(nUnique, s);
    if (nUnique)
        kRestrictWeights<<<grid(nUnique), TPB, 0, s>>>(nUnique, S.faceBeg.p, S.faceEnd.p, S.faceList.p, w, cw.p);
    B2G_LAUNCH_CHECK();
    // internal faces grouped by coarse cell, ascending
    const int nInternal = nF - nValid;
    S.intStart.alloc(nC + 1, s);
    S.intList.alloc(nInternal, s);
    {
        DBuf<unsigned> ik, iks;
        ik.alloc(nInternal, s);
        iks.alloc(nInternal, s);
        if (nInternal)
            kInternalKeys<<<grid(nInternal), TPB, 0, s>>>(nInternal, faces.p + nValid, S.faceRestrict.p, ik.p);
        B2G_LAUNCH_CHECK();
        sortPairs(ik.p, iks.p, faces.p + nValid, S.intList.p, nInternal, cbits, s);
        DBuf<int> ikInt;
        ikInt.alloc(nInternal, s);
        if (nInternal) kKeysToInt<<<grid(nInternal), TPB, 0, s>>>(nInternal, iks.p, ikInt.p);
        countingStarts(ikInt.p, nInternal, nC, S.intStart.p, s);
    }
    // fine cells grouped by coarse cell, ascending
    S.cellStart.alloc(nC + 1, s);
    S.cellList.alloc(S.nFine, s);
    {
        DBuf<int> ci;
        DBuf<unsigned> ck;
        ci.alloc(S.nFine, s);
        ck.alloc(S.nFine, s);
        kIota<<<grid(S.nFine), TPB, 0, s>>>(ci.p, S.nFine);
        B2G_LAUNCH_CHECK();
        sortPairs(reinterpret_cast<const unsigned*>(S.restrictAddr.p), ck.p, ci.p, S.cellList.p, S.nFine,
                  cbits, s);
        countingStarts(S.restrictAddr.p, S.nFine, nC, S.cellStart.p, s);
    }
}

void buildHierarchy(Mesh& M, const double* dSf, const double* dMagSf, int nCellsInCoarsestLevel,
                    int* forward)
{
    cudaStream_t s = M.stream;
    LevelAddr& L0 = M.lev[0];
    buildLevelLayouts(L0, s);
    // GAMGAgglomeration.C:285 (AGG:297)
    int nCoarsest = std::min(L0.nCells / 2, nCellsInCoarsestLevel);
    nCoarsest = std::max(1, nCoarsest);
    DBuf<double> w;
    w.alloc(L0.nFaces, s);
    if (L0.nFaces) kFaceWeights<<<grid(L0.nFaces), TPB, 0, s>>>(L0.nFaces, dSf, dMagSf, w.p);
    B2G_LAUNCH_CHECK();
    int fwd = *forward ? 1 : 0;
    while (static_cast<int>(M.step.size()) < kMaxLevels - 1)
    {
        LevelAddr& F = M.lev.back();
        DBuf<int> map;
        const int nCoarse = pairPass(F, w.p, fwd, map, s);
        fwd = !fwd;  // flips after every pass, the rejected one included (AGG:282)
        // continueAgglomerating (AGG:17-24)
        if (nCoarse < nCoarsest || !(nCoarse < F.nCells)) break;
        M.step.emplace_back();
        Step& S = M.step.back();
        S.nFine = F.nCells;
        S.nCoarse = nCoarse;
        S.nFineFaces = F.nFaces;
        S.restrictAddr = std::move(map);
        M.lev.emplace_back();
        LevelAddr& Fr = M.lev[M.lev.size() - 2];
        LevelAddr& Cl = M.lev.back();
        DBuf<double> cw;
        coarseAddressing(Fr, S, Cl, w.p, cw, s);
        buildLevelLayouts(Cl, s);
        w = std::move(cw);
    }
    *forward = fwd;
    for (auto& L : M.lev) buildGsSchedule(L, s);
    for (int i = 0; i < M.nLevels(); ++i) buildStepMaps(M, i);
}

void buildHierarchyFromMaps(Mesh& M, const double* dSf, const double* dMagSf,
                            const std::vector<std::vector<int>>& maps, const std::vector<int>& nCoarse)
{
    cudaStream_t s = M.stream;
    LevelAddr& L0 = M.lev[0];
    buildLevelLayouts(L0, s);
    DBuf<double> w;
    w.alloc(std::max(L0.nFaces, 1), s);
    if (L0.nFaces) kFaceWeights<<<grid(L0.nFaces), TPB, 0, s>>>(L0.nFaces, dSf, dMagSf, w.p);
    B2G_LAUNCH_CHECK();
    for (size_t i = 0; i < maps.size(); ++i)
    {
        LevelAddr& F = M.lev.back();
        if (static_cast<int>(maps[i].size()) != F.nCells)
            fail(B2G_ERR_STATE, "b2g: the cached hierarchy does not fit this mesh (restriction map size).");
        M.step.emplace_back();
        Step& S = M.step.back();
        S.nFine = F.nCells;
        S.nCoarse = nCoarse[i];
        S.nFineFaces = F.nFaces;
        S.restrictAddr.upload(maps[i].data(), maps[i].size(), s);
        M.lev.emplace_back();
        LevelAddr& Fr = M.lev[M.lev.size() - 2];
        LevelAddr& Cl = M.lev.back();
        DBuf<double> cw;
        coarseAddressing(Fr, S, Cl, w.p, cw, s);
        buildLevelLayouts(Cl, s);
        w = std::move(cw);
    }
    for (auto& L : M.lev) buildGsSchedule(L, s);
    for (int i = 0; i < M.nLevels(); ++i) buildStepMaps(M, i);
}


// ---------------------------------------------------------------------------------------------
// Gauss-Seidel schedule
// ---------------------------------------------------------------------------------------------

void buildEll(GsSchedule& G, int n, cudaStream_t s);

void buildGsSchedule(LevelAddr& L, cudaStream_t s)
{
    GsSchedule& G = L.gs;
    const int n = L.nCells;
    G.depth.alloc(n, s);
    if (n == 0) return;
    // depths by Kahn's frontier: a cell's depth is one more than its deepest owner-side neighbour
    {
        DBuf<int> indeg, fa, fb, sizes;
        indeg.alloc(n, s);
        fa.alloc(n, s);
        fb.alloc(n, s);
        sizes.alloc(2, s);
        sizes.zero(s);
        kIndegree<<<grid(n), TPB, 0, s>>>(n, L.losortStart.p, indeg.p, fa.p, sizes.p);
        B2G_LAUNCH_CHECK();
        int fsize = readInt(sizes.p, s);
        int round = 0;
        int done = 0;
        int* cur = fa.p;
        int* nxt = fb.p;
        int hsz[2];
        while (fsize > 0)
        {
            done += fsize;
            B2G_CUDA(cudaMemsetAsync(sizes.p + 1, 0, sizeof(int), s));
            kDepthRound<<<grid(fsize), TPB, 0, s>>>(round, cur, fsize, L.ownStart.p, L.upper.p, indeg.p,
                                                    G.depth.p, nxt, sizes.p + 1);
            B2G_LAUNCH_CHECK();
            B2G_CUDA(cudaMemcpyAsync(hsz, sizes.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
            B2G_CUDA(cudaStreamSynchronize(s));
            fsize = hsz[1];
            std::swap(cur, nxt);
            ++round;
        }
        if (done != n) fail(B2G_ERR_STATE, "b2g: the Gauss-Seidel dependency graph has a cycle.");
        G.maxDepth = round - 1;
    }
    // parts: contiguous cell ranges balanced by row length; enough of them to fill the GPU when a
    // depth holds many cells, one when the level is narrow (a single CTA then walks it). One part per
    // g_partCells cells of the average depth, 48 by default: measured on B200 against 16, 24, 32,
    // 128, 384 and 1024 (graded 128^3 and 272^3 solves), more parts shorten each part's chain more
    // than the hand-offs cost. A batch, whose cases fill the GPU together, is faster with 128.
    const int depthCount = G.maxDepth + 1;
    const long long avgPerDepth = (static_cast<long long>(n) + depthCount - 1) / depthCount;
    const int nSM = DeviceInfo::get().numSMs;
    int P = static_cast<int>(std::min<long long>(nSM, std::max<long long>(1, avgPerDepth / g_partCells.load())));
    if (n < 4096) P = 1;
    G.nParts = P;
    if (n >= (1 << 30)) fail(B2G_ERR_ARGUMENT, "b2g: a level of 2^30 cells or more does not fit the sweep's codes.");
    DBuf<int> dPartStart, partOf;
    dPartStart.alloc(P + 1, s);
    kPartBounds<<<grid(P + 1), TPB, 0, s>>>(n, P, L.rowStart.p, dPartStart.p);
    partOf.alloc(n, s);
    kPartOf<<<grid(n), TPB, 0, s>>>(n, P, dPartStart.p, partOf.p);
    const int stride = G.maxDepth + 1;
    if (static_cast<long long>(P) * stride >= (1LL << 32))
        fail(B2G_ERR_ARGUMENT, "b2g: the Gauss-Seidel schedule is too deep for its 32-bit keys.");
    DBuf<unsigned> keys, skeys;
    DBuf<int> iota;
    keys.alloc(n, s);
    skeys.alloc(n, s);
    iota.alloc(n, s);
    kSchedKeys<<<grid(n), TPB, 0, s>>>(n, stride, partOf.p, G.depth.p, keys.p);
    kIota<<<grid(n), TPB, 0, s>>>(iota.p, n);
    B2G_LAUNCH_CHECK();
    G.posCell.alloc(n, s);
    sortPairs(keys.p, skeys.p, iota.p, G.posCell.p, n, bitsFor(static_cast<long long>(P) * stride), s);
    // (part, depth) groups
    DBuf<int> head, lvlScan;
    head.alloc(n, s);
    lvlScan.alloc(n + 1, s);
    kKeyHeads<<<grid(n), TPB, 0, s>>>(n, skeys.p, head.p);
    B2G_LAUNCH_CHECK();
    const int nLvl = static_cast<int>(exclusiveScan(head.p, lvlScan.p, n, s));
    DBuf<int> lvlStart, lvlDepth, lvlPart;
    lvlStart.alloc(nLvl, s);
    lvlDepth.alloc(nLvl, s);
    lvlPart.alloc(nLvl, s);
    kLevelInfo<<<grid(n), TPB, 0, s>>>(n, stride, skeys.p, head.p, lvlScan.p, lvlStart.p, lvlDepth.p, lvlPart.p);
    B2G_LAUNCH_CHECK();
    // row layout in position order
    DBuf<int> rowLen;
    G.posOf.alloc(n, s);
    rowLen.alloc(n, s);
    kPosOf<<<grid(n), TPB, 0, s>>>(n, G.posCell.p, G.posOf.p);
    kPosRowLen<<<grid(n), TPB, 0, s>>>(n, G.posCell.p, L.rowStart.p, rowLen.p);
    B2G_LAUNCH_CHECK();
    G.posRow.alloc(n + 1 + 8, s);
    G.posRow.zero(s);
    exclusiveScan(rowLen.p, G.posRow.p, n, s);
    G.entColPos.alloc(std::max<size_t>(2 * (size_t)L.nFaces, 1), s);
    G.entFacePos.alloc(std::max<size_t>(2 * (size_t)L.nFaces, 1), s);
    kCsrPositions<<<grid(n), TPB, 0, s>>>(n, G.posCell.p, G.posOf.p, L.rowStart.p, L.col.p, L.entFace.p, G.posRow.p,
                                          G.entColPos.p, G.entFacePos.p);
    B2G_LAUNCH_CHECK();
    // chunks: each (part, depth) group cut into chunks of at most M cells and E sliced-ELL entries
    const std::vector<int> hLvlStart = lvlStart.download(s);
    const std::vector<int> hLvlDepth = lvlDepth.download(s);
    const std::vector<int> hLvlPart = lvlPart.download(s);
    const std::vector<int> hPosRow = G.posRow.download(s);
    int maxGroup = 0, maxRow = 0;
    for (int g = 0; g < nLvl; ++g)
        maxGroup = std::max(maxGroup, (g + 1 < nLvl ? hLvlStart[g + 1] : n) - hLvlStart[g]);
    for (int i = 0; i < n; ++i) maxRow = std::max(maxRow, hPosRow[i + 1] - hPosRow[i]);
    if (maxRow > 255) fail(B2G_ERR_ARGUMENT, "b2g: a cell with more than 255 faces does not fit the sweep's rows.");
    const int nnz = hPosRow[n];
    const int rowCap = std::max(1, std::min(maxRow, static_cast<int>((5LL * nnz + 4LL * n - 1) / (4LL * n))));
    const size_t smemCap = 200 * 1024;
    auto fits = [&](int m, int e, int g) {
        int ah, bh;
        k::gsWindowExtents(m, ah, bh);
        return k::gsSmemBytes<double>(m, e, g) <= smemCap && ah >= m && bh >= m &&
               k::kWin + k::kStages * g + 1 <= k::kMaxTable;
    };
    const int words = (P + 31) / 32;
    int M = std::min(k::kMaxCompute, std::max(32, ((maxGroup + 31) / 32) * 32));
    const EntryClass ecBase{k::kWin, 0, 0, partOf.p, nullptr, nullptr};
    for (int attempt = 0;; ++attempt)
    {
        // entry budget: the average row (plus a margin) per cell, at least one slice of the longest row
        int E = std::max(M * rowCap, 32 * maxRow);
        E = ((E + 31) / 32) * 32;
        while (M > 32 && !fits(M, E, M)) { M -= 32; E = ((std::max(M * rowCap, 32 * maxRow) + 31) / 32) * 32; }
        if (!fits(M, E, 32)) fail(B2G_ERR_ARGUMENT, "b2g: a cell has more faces than the Gauss-Seidel pipeline holds.");
        // host chunking: per chunk its positions and ELL entries; per position its row descriptor
        std::vector<int> hChunkStart, hChunkDepth, hChunkNewDepth, hPartChunk(P + 1, 0);
        std::vector<long long> hChunkEnt0;
        std::vector<unsigned> hPosEnt(static_cast<size_t>(n) + 8, 0u);
        long long ent = 0;
        int prevPart = -1;
        for (int g = 0; g < nLvl; ++g)
        {
            const int gs = hLvlStart[g];
            const int ge = g + 1 < nLvl ? hLvlStart[g + 1] : n;
            int cs = gs;
            while (cs < ge)
            {
                // grow the chunk slice by slice (32 cells, padded to the slice's longest row)
                int ce = cs;
                long long nEnt = 0;
                while (ce < ge && ce - cs < M)
                {
                    const int sEnd = std::min({ce + 32, ge, cs + M});
                    int w = 0;
                    for (int i = ce; i < sEnd; ++i) w = std::max(w, hPosRow[i + 1] - hPosRow[i]);
                    if (nEnt + 32LL * w > E && ce > cs) break;
                    for (int i = ce; i < sEnd; ++i)
                        hPosEnt[i] = (static_cast<unsigned>(w) << 24) | static_cast<unsigned>(nEnt + (i - ce));
                    nEnt += 32LL * w;
                    ce = sEnd;
                }
                hChunkStart.push_back(cs);
                hChunkEnt0.push_back(ent);
                hChunkDepth.push_back(hLvlDepth[g]);
                hChunkNewDepth.push_back(cs == gs && prevPart == hLvlPart[g] ? 1 : 0);
                hPartChunk[hLvlPart[g] + 1]++;
                prevPart = hLvlPart[g];
                ent += nEnt;
                cs = ce;
            }
        }
        const int nCh = static_cast<int>(hChunkStart.size());
        hChunkStart.push_back(n);
        hChunkEnt0.push_back(ent);
        for (int q = 0; q < P; ++q) hPartChunk[q + 1] += hPartChunk[q];
        int ahead, behind;
        k::gsWindowExtents(M, ahead, behind);
        // device classification
        DBuf<int> chunkStart, chunkDepth, chunkNewDepth, chunkNeedUp, chunkSameWait, chunkOf;
        DBuf<int> cntOld, cntNew, oldOff, newOff;
        DBuf<long long> chunkEnt0;
        chunkStart.upload(hChunkStart.data(), hChunkStart.size(), s);
        chunkDepth.upload(hChunkDepth.data(), hChunkDepth.size(), s);
        chunkNewDepth.upload(hChunkNewDepth.data(), hChunkNewDepth.size(), s);
        chunkEnt0.upload(hChunkEnt0.data(), hChunkEnt0.size(), s);
        G.posEnt.upload(hPosEnt.data(), hPosEnt.size(), s);
        chunkNeedUp.alloc(nCh, s);
        chunkSameWait.alloc(nCh, s);
        kFillInt<<<grid(nCh), TPB, 0, s>>>(chunkNeedUp.p, nCh, -1);
        kFillInt<<<grid(nCh), TPB, 0, s>>>(chunkSameWait.p, nCh, -1);
        chunkOf.alloc(n, s);
        kChunkOfPos<<<grid(n), TPB, 0, s>>>(n, nCh, chunkStart.p, chunkOf.p);
        DBuf<unsigned> upBits;
        upBits.alloc(static_cast<size_t>(P) * words, s);
        upBits.zero(s);
        EntryClass ec = ecBase;
        ec.ahead = ahead;
        ec.behind = behind;
        ec.chunkOf = chunkOf.p;
        ec.chunkStart = chunkStart.p;
        cntOld.alloc(n, s);
        cntNew.alloc(n, s);
        kGatherCounts<<<grid(n), TPB, 0, s>>>(n, ec, G.posCell.p, G.posOf.p, G.depth.p, L.rowStart.p,
                                              L.losortStart.p, L.col.p, cntOld.p, cntNew.p, chunkNeedUp.p,
                                              chunkSameWait.p, upBits.p, words);
        B2G_LAUNCH_CHECK();
        oldOff.alloc(n + 1, s);
        newOff.alloc(n + 1, s);
        const long long nGather = exclusiveScan(cntOld.p, oldOff.p, n, s) + exclusiveScan(cntNew.p, newOff.p, n, s);
        // the largest gather list of a chunk sizes the slots' gather arrays
        const std::vector<int> hOldOff = oldOff.download(s);
        const std::vector<int> hNewOff = newOff.download(s);
        int maxGat = 0;
        for (int c = 0; c < nCh; ++c)
            maxGat = std::max(maxGat, hOldOff[hChunkStart[c + 1]] - hOldOff[hChunkStart[c]] +
                                          hNewOff[hChunkStart[c + 1]] - hNewOff[hChunkStart[c]]);
        maxGat = ((maxGat + 1) / 2) * 2;
        if (!fits(M, E, maxGat) && M > 32 && attempt < 16)
        {
            M -= 32;  // fewer cells per chunk: fewer gathers per chunk, and more room per slot
            continue;
        }
        if (!fits(M, E, maxGat))
            fail(B2G_ERR_ARGUMENT, "b2g: the Gauss-Seidel chunks gather more values than shared memory holds.");
        G.maxCells = M;
        G.maxEnt = E;
        G.maxGat = maxGat;
        G.ahead = ahead;
        G.behind = behind;
        G.nChunks = nCh;
        G.nEll = ent;
        G.nGather = nGather;
        G.nPadded = ((n + k::kFill - 1) / k::kFill) * k::kFill;
        G.nAlloc = G.nPadded + k::kFill;
        G.partChunkStart.upload(hPartChunk.data(), hPartChunk.size(), s);
        G.gsCode.alloc(std::max<long long>(ent, 1), s);
        G.gsEntFace.alloc(std::max<long long>(ent, 1), s);
        G.gatSrc.alloc(std::max<long long>(nGather, 1) + 8, s);  // + the 16-byte cover of a bulk copy
        if (ent)
        {
            // padding entries read the table's zero
            kFillShort<<<std::min<long long>(ceilDiv(ent, TPB), 8192), TPB, 0, s>>>(
                G.gsCode.p, ent, static_cast<unsigned short>(k::kWin + k::kStages * maxGat));
            kFillInt<<<static_cast<int>(std::min<long long>(ceilDiv(ent, TPB), 1LL << 30)), TPB, 0, s>>>(
                G.gsEntFace.p, static_cast<int>(ent), -1);
        }
        kSweepEntries<<<grid(n), TPB, 0, s>>>(n, ec, maxGat, G.partChunkStart.p, G.posCell.p, G.posOf.p, L.rowStart.p,
                                              L.losortStart.p, L.col.p, L.entFace.p, G.posEnt.p, chunkEnt0.p, oldOff.p,
                                              newOff.p, G.gsCode.p, G.gsEntFace.p, G.gatSrc.p);
        B2G_LAUNCH_CHECK();
        // each chunk's blob offset (16-byte units) in the FP64 and the FP32 blobs
        std::vector<int2> hBlob(nCh);
        long long b64 = 0, b32 = 0;
        for (int c = 0; c < nCh; ++c)
        {
            const int m = hChunkStart[c + 1] - hChunkStart[c];
            const int ne = static_cast<int>(hChunkEnt0[c + 1] - hChunkEnt0[c]);
            hBlob[c] = make_int2(static_cast<int>(b64 / 16), static_cast<int>(b32 / 16));
            b64 += k::blobLayout<double>(m, ne).bytes;
            b32 += k::blobLayout<float>(m, ne).bytes;
        }
        if (b64 / 16 >= (1LL << 31)) fail(B2G_ERR_ARGUMENT, "b2g: the level's sweep data exceeds 32 GiB.");
        G.blobBytes64 = b64;
        G.blobBytes32 = b32;
        DBuf<int2> chunkBlob;
        chunkBlob.upload(hBlob.data(), hBlob.size(), s);
        G.chunkRec.alloc(12 * (size_t)nCh, s);
        kChunkRecs<<<grid(nCh), TPB, 0, s>>>(nCh, chunkStart.p, chunkEnt0.p, chunkDepth.p, chunkNewDepth.p, oldOff.p,
                                             newOff.p, chunkNeedUp.p, chunkSameWait.p, chunkBlob.p, G.chunkRec.p);
        B2G_LAUNCH_CHECK();
        // upstream parts (whose progress a part waits on) and which parts have a downstream
        std::vector<unsigned> hUp = upBits.download(s);
        std::vector<int> upStart(P + 1, 0), upList;
        for (int q = 0; q < P; ++q)
        {
            upStart[q] = static_cast<int>(upList.size());
            for (int r = 0; r < P; ++r)
                if (hUp[(size_t)q * words + (r >> 5)] & (1u << (r & 31))) upList.push_back(r);
        }
        upStart[P] = static_cast<int>(upList.size());
        std::vector<int> hasDown(P, 0);
        for (int r : upList) hasDown[r] = 1;
        G.hasDown.upload(hasDown.data(), hasDown.size(), s);
        G.upStart.upload(upStart.data(), upStart.size(), s);
        if (upList.empty()) upList.push_back(0);
        G.upList.upload(upList.data(), upList.size(), s);
        B2G_CUDA(cudaStreamSynchronize(s));
        break;
    }
    G.partPosStart = std::move(dPartStart);
    // the parts' progress lines, then one line for a launch's ticket counter
    G.progress.alloc(static_cast<size_t>(P + 1) * k::kProgressStride, s);
    G.progress.zero(s);
    if (n >= kEllMinCells) buildEll(G, n, s);
    B2G_CUDA(cudaStreamSynchronize(s));
}

// the sliced ELL copy of a level's position-order rows (ldu_kernels.cuh Rows)
void buildEll(GsSchedule& G, int n, cudaStream_t s)
{
    const int nSlices = (n + 31) / 32;
    DBuf<int> width32;
    width32.alloc(nSlices, s);
    kEllWidth<<<grid(nSlices), TPB, 0, s>>>(n, nSlices, G.posRow.p, width32.p);
    B2G_LAUNCH_CHECK();
    G.ellBase.alloc(static_cast<size_t>(nSlices) + 1, s);
    const long long nEnt = exclusiveScan(width32.p, G.ellBase.p, nSlices, s);
    if (nEnt >= (1LL << 31)) fail(B2G_ERR_ARGUMENT, "b2g: a level's sliced rows exceed 2^31 entries.");
    G.nEllEnt = nEnt;
    G.ellCol.alloc(std::max<long long>(nEnt, 1), s);
    G.ellEnt.alloc(std::max<long long>(nEnt, 1), s);
    kEllFill<<<grid(nSlices * 32LL), TPB, 0, s>>>(n, G.posRow.p, G.entColPos.p, G.ellBase.p, G.ellCol.p, G.ellEnt.p);
    B2G_LAUNCH_CHECK();
}

namespace {

// greedy colouring, one depth group at a time: a cell's neighbours of smaller depth are coloured,
// those of larger depth not yet, and cells of one depth share no face; the cell takes the smallest
// colour its coloured neighbours do not have
__global__ void kColourDepth(int b, int e, const int* __restrict__ byDepth, const int* __restrict__ rowStart,
                             const int* __restrict__ col, int* __restrict__ colour, int* __restrict__ err)
{
    const int i = b + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= e) return;
    const int c = byDepth[i];
    unsigned long long used = 0ull;
    for (int q = rowStart[c]; q < rowStart[c + 1]; ++q)
    {
        const int k = colour[col[q]];
        if (k >= 0) used |= 1ull << k;
    }
    if (used == ~0ull)
    {
        atomicOr(err, 1);
        colour[c] = 63;
        return;
    }
    colour[c] = __ffsll(static_cast<long long>(~used)) - 1;
}

__global__ void kCheckColours(int nF, const int* __restrict__ lower, const int* __restrict__ upper,
                              const int* __restrict__ colour, int* __restrict__ err, int* __restrict__ maxColour)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    const int a = colour[lower[f]], b = colour[upper[f]];
    if (a == b || a < 0 || b < 0) atomicOr(err, 2);
    atomicMax(maxColour, max(a, b));
}

__global__ void kColourOfPos(int n, const int* __restrict__ posCell, const int* __restrict__ colour,
                             unsigned* __restrict__ key, int* __restrict__ iota, int* __restrict__ maxColour)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int k = colour[posCell[p]];
    key[p] = static_cast<unsigned>(k);
    iota[p] = p;
    atomicMax(maxColour, k);
}

// the colour-major rows: sorted position i of colour k goes to padded row padStart[k] + i - start[k]
__global__ void kScatterRows(int n, const unsigned* __restrict__ sortedKey, const int* __restrict__ sortedPos,
                             const int* __restrict__ start, const int* __restrict__ padStart, int* __restrict__ rowPos)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = static_cast<int>(sortedKey[i]);
    rowPos[padStart[k] + i - start[k]] = sortedPos[i];
}

// a slice's width: the longest row of its 32
__global__ void kSliceWidth(int nSlices, const int* __restrict__ rowPos, const int* __restrict__ posCell,
                            const int* __restrict__ rowStart, int* __restrict__ width32)
{
    const int sl = blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= nSlices) return;
    int w = 0;
    for (int l = 0; l < 32; ++l)
    {
        const int p = rowPos[32 * sl + l];
        if (p >= 0)
        {
            const int c = posCell[p];
            w = max(w, rowStart[c + 1] - rowStart[c]);
        }
    }
    width32[sl] = 32 * w;
}

__global__ void kFillSlices(int nRows, const int* __restrict__ rowPos, const int* __restrict__ sliceBase,
                            const int* __restrict__ posCell, const int* __restrict__ posOf,
                            const int* __restrict__ rowStart, const int* __restrict__ col,
                            const int* __restrict__ entFace, int* __restrict__ colP, int* __restrict__ faceP)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nRows) return;
    const int sl = r >> 5, lane = r & 31;
    const int base = sliceBase[sl];
    const int w = (sliceBase[sl + 1] - base) >> 5;
    const int p = rowPos[r];
    const int c = p >= 0 ? posCell[p] : -1;
    const int len = c >= 0 ? rowStart[c + 1] - rowStart[c] : 0;
    for (int q = 0; q < w; ++q)
    {
        const int e = base + 32 * q + lane;
        if (q < len)
        {
            colP[e] = posOf[col[rowStart[c] + q]];
            faceP[e] = entFace[rowStart[c] + q];
        }
        else
        {
            colP[e] = p >= 0 ? p : 0;  // reads a value with coefficient zero
            faceP[e] = -1;
        }
    }
}

}  // namespace

// On the device: greedy colouring in depth order (a structured hex level gets a checkerboard's two
// colours), checked face by face; then the colour-major sliced-ELL rows in position order.
void buildColouring(LevelAddr& L, cudaStream_t s)
{
    Colouring& C = L.mc;
    if (C.nColours > 0) return;
    const int n = L.nCells, nF = L.nFaces;
    const GsSchedule& G = L.gs;
    DBuf<int> colour, byDepth, depthStart, err, maxC;
    colour.alloc(std::max(n, 1), s);
    kFillInt<<<grid(n), TPB, 0, s>>>(colour.p, n, -1);
    err.alloc(1, s);
    err.zero(s);
    maxC.alloc(1, s);
    maxC.zero(s);
    {
        DBuf<int> iota;
        DBuf<unsigned> kout;
        iota.alloc(std::max(n, 1), s);
        kout.alloc(std::max(n, 1), s);
        byDepth.alloc(std::max(n, 1), s);
        kIota<<<grid(n), TPB, 0, s>>>(iota.p, n);
        B2G_LAUNCH_CHECK();
        sortPairs(reinterpret_cast<const unsigned*>(G.depth.p), kout.p, iota.p, byDepth.p, n, bitsFor(G.maxDepth + 1), s);
        depthStart.alloc(G.maxDepth + 2, s);
        countingStarts(G.depth.p, n, G.maxDepth + 1, depthStart.p, s);
    }
    const std::vector<int> hDepth = depthStart.download(s);
    for (int d = 0; d <= G.maxDepth; ++d)
    {
        const int b = hDepth[d], e = hDepth[d + 1];
        if (e > b) kColourDepth<<<grid(e - b), TPB, 0, s>>>(b, e, byDepth.p, L.rowStart.p, L.col.p, colour.p, err.p);
    }
    B2G_LAUNCH_CHECK();
    if (nF) kCheckColours<<<grid(nF), TPB, 0, s>>>(nF, L.lower.p, L.upper.p, colour.p, err.p, maxC.p);
    B2G_LAUNCH_CHECK();
    const int e = readInt(err.p, s);
    if (e & 1) fail(B2G_ERR_ARGUMENT, "b2g: a level needs more than 63 colours for the multicolour sweep.");
    if (e & 2) fail(B2G_ERR_STATE, "b2g: the multicolour layout has two neighbours of one colour.");
    // positions by colour, ascending within a colour (stable sort)
    DBuf<unsigned> key, skey;
    DBuf<int> iota, spos;
    key.alloc(std::max(n, 1), s);
    skey.alloc(std::max(n, 1), s);
    iota.alloc(std::max(n, 1), s);
    spos.alloc(std::max(n, 1), s);
    if (n) kColourOfPos<<<grid(n), TPB, 0, s>>>(n, G.posCell.p, colour.p, key.p, iota.p, maxC.p);
    B2G_LAUNCH_CHECK();
    const int nColours = readInt(maxC.p, s) + 1;
    sortPairs(key.p, skey.p, iota.p, spos.p, n, bitsFor(nColours), s);
    DBuf<int> start;
    start.alloc(nColours + 1, s);
    countingStarts(reinterpret_cast<const int*>(key.p), n, nColours, start.p, s);
    const std::vector<int> hStart = start.download(s);
    C.colourStart.assign(1, 0);
    for (int k = 0; k < nColours; ++k)
        C.colourStart.push_back(C.colourStart.back() + ((hStart[k + 1] - hStart[k] + 31) / 32) * 32);
    C.nRows = C.colourStart.back();
    C.colourStartD.upload(C.colourStart.data(), C.colourStart.size(), s);
    C.pos.alloc(std::max(C.nRows, 1), s);
    kFillInt<<<grid(std::max(C.nRows, 1)), TPB, 0, s>>>(C.pos.p, std::max(C.nRows, 1), -1);
    if (n) kScatterRows<<<grid(n), TPB, 0, s>>>(n, skey.p, spos.p, start.p, C.colourStartD.p, C.pos.p);
    B2G_LAUNCH_CHECK();
    const int nSlices = C.nRows / 32;
    DBuf<int> width32;
    width32.alloc(std::max(nSlices, 1), s);
    if (nSlices) kSliceWidth<<<grid(nSlices), TPB, 0, s>>>(nSlices, C.pos.p, G.posCell.p, L.rowStart.p, width32.p);
    B2G_LAUNCH_CHECK();
    C.sliceBase.alloc(nSlices + 1, s);
    const long long nEnt = exclusiveScan(width32.p, C.sliceBase.p, nSlices, s);
    if (nEnt >= (1LL << 31)) fail(B2G_ERR_ARGUMENT, "b2g: the multicolour layout exceeds 2^31 entries.");
    C.nEnt = nEnt;
    C.col.alloc(std::max<long long>(nEnt, 1), s);
    C.face.alloc(std::max<long long>(nEnt, 1), s);
    if (nEnt == 0)
    {
        kFillInt<<<1, 1, 0, s>>>(C.col.p, 1, 0);
        kFillInt<<<1, 1, 0, s>>>(C.face.p, 1, -1);
    }
    if (C.nRows)
        kFillSlices<<<grid(C.nRows), TPB, 0, s>>>(C.nRows, C.pos.p, C.sliceBase.p, G.posCell.p, G.posOf.p,
                                                  L.rowStart.p, L.col.p, L.entFace.p, C.col.p, C.face.p);
    B2G_LAUNCH_CHECK();
    B2G_CUDA(cudaStreamSynchronize(s));
    C.nColours = nColours;
}

namespace {

// the reversed faces: face f' is losort[nF-1-f'] (neighbours descending, faces descending within
// one), owner' = n-1-neighbour, neighbour' = n-1-owner: again sorted by owner'
__global__ void kRevFaces(int nF, int nC, const int* __restrict__ losort, const int* __restrict__ lower,
                          const int* __restrict__ upper, int* __restrict__ rl, int* __restrict__ ru)
{
    const int f2 = blockIdx.x * blockDim.x + threadIdx.x;
    if (f2 >= nF) return;
    const int f = losort[nF - 1 - f2];
    rl[f2] = nC - 1 - upper[f];
    ru[f2] = nC - 1 - lower[f];
}

// the reversed rows: for cell c' = n-1-c, the faces c owns in ascending face order (the order in
// which the backward walk subtracts them), the other cell in reversed numbering
__global__ void kRevRows(int nC, const int* __restrict__ ownStart, const int* __restrict__ upper,
                         const int* __restrict__ rowStartR, int* __restrict__ colR, int* __restrict__ faceR,
                         int descending)
{
    const int c2 = blockIdx.x * blockDim.x + threadIdx.x;
    if (c2 >= nC) return;
    const int c = nC - 1 - c2;
    int k = rowStartR[c2];
    const int f0 = ownStart[c], f1 = ownStart[c + 1];
    for (int i = 0; i < f1 - f0; ++i)
    {
        const int f = descending ? f1 - 1 - i : f0 + i;
        colR[k] = nC - 1 - upper[f];
        faceR[k] = f;
        ++k;
    }
}

// the lower-only rows: the faces the cell is the neighbour of, ascending (losort order)
__global__ void kLowerRows(int nC, const int* __restrict__ losortStart, const int* __restrict__ losort,
                           const int* __restrict__ lower, int* __restrict__ col, int* __restrict__ face)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    for (int q = losortStart[c]; q < losortStart[c + 1]; ++q)
    {
        col[q] = lower[losort[q]];
        face[q] = losort[q];
    }
}

__global__ void kSamePos(int n, const int* __restrict__ posCellF, const int* __restrict__ posOfR,
                         int* __restrict__ outPos)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) outPos[p] = posOfR[posCellF[p]];
}

__global__ void kRevPos(int n, const int* __restrict__ posCellF, const int* __restrict__ posOfR,
                        int* __restrict__ revPos)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) revPos[p] = posOfR[n - 1 - posCellF[p]];
}

}  // namespace

void buildReversedLevel(LevelAddr& L, cudaStream_t s, bool descending)
{
    if (descending ? static_cast<bool>(L.revDesc) : static_cast<bool>(L.rev)) return;
    const int n = L.nCells, nF = L.nFaces;
    std::unique_ptr<LevelAddr> R(new LevelAddr);
    R->nCells = n;
    R->nFaces = nF;
    R->lower.alloc(std::max(nF, 1), s);
    R->upper.alloc(std::max(nF, 1), s);
    if (nF) kRevFaces<<<grid(nF), TPB, 0, s>>>(nF, n, L.losort.p, L.lower.p, L.upper.p, R->lower.p, R->upper.p);
    B2G_LAUNCH_CHECK();
    buildLevelLayouts(*R, s);
    // rows of the own faces only: the counts are the reversed level's neighbour counts
    B2G_CUDA(cudaMemcpyAsync(R->rowStart.p, R->losortStart.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice, s));
    if (n)
        kRevRows<<<grid(n), TPB, 0, s>>>(n, L.ownStart.p, L.upper.p, R->rowStart.p, R->col.p, R->entFace.p,
                                         descending ? 1 : 0);
    B2G_LAUNCH_CHECK();
    buildGsSchedule(*R, s);
    DBuf<int>& pos = descending ? L.revDescPos : L.revPos;
    pos.alloc(std::max(n, 1), s);
    if (n) kRevPos<<<grid(n), TPB, 0, s>>>(n, L.gs.posCell.p, R->gs.posOf.p, pos.p);
    B2G_LAUNCH_CHECK();
    B2G_CUDA(cudaStreamSynchronize(s));
    (descending ? L.revDesc : L.rev) = std::move(R);
}

void buildLowerLevel(LevelAddr& L, cudaStream_t s)
{
    if (L.lowerOnly) return;
    const int n = L.nCells, nF = L.nFaces;
    std::unique_ptr<LevelAddr> R(new LevelAddr);
    R->nCells = n;
    R->nFaces = nF;
    R->lower.alloc(std::max(nF, 1), s);
    R->upper.alloc(std::max(nF, 1), s);
    if (nF)
    {
        B2G_CUDA(cudaMemcpyAsync(R->lower.p, L.lower.p, sizeof(int) * nF, cudaMemcpyDeviceToDevice, s));
        B2G_CUDA(cudaMemcpyAsync(R->upper.p, L.upper.p, sizeof(int) * nF, cudaMemcpyDeviceToDevice, s));
    }
    buildLevelLayouts(*R, s);
    B2G_CUDA(cudaMemcpyAsync(R->rowStart.p, R->losortStart.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice, s));
    if (n) kLowerRows<<<grid(n), TPB, 0, s>>>(n, R->losortStart.p, R->losort.p, R->lower.p, R->col.p, R->entFace.p);
    B2G_LAUNCH_CHECK();
    buildGsSchedule(*R, s);
    L.lowerPos.alloc(std::max(n, 1), s);
    if (n) kSamePos<<<grid(n), TPB, 0, s>>>(n, L.gs.posCell.p, R->gs.posOf.p, L.lowerPos.p);
    B2G_LAUNCH_CHECK();
    B2G_CUDA(cudaStreamSynchronize(s));
    L.lowerOnly = std::move(R);
}

namespace {
__global__ void kEllColCoarse(long long nEnt, const int* __restrict__ ellCol, const int* __restrict__ prolongP,
                              int* __restrict__ out)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nEnt; e += (long long)gridDim.x * blockDim.x)
    {
        const int c = ellCol[e];
        out[e] = c >= 0 ? prolongP[c] : -1;
    }
}
}  // namespace

void buildStepMaps(Mesh& M, int i)
{
    cudaStream_t s = M.stream;
    Step& S = M.step[i];
    const GsSchedule& F = M.lev[i].gs;
    const GsSchedule& C = M.lev[i + 1].gs;
    DBuf<int> cnt;
    cnt.alloc(S.nCoarse, s);
    kStepCounts<<<grid(S.nCoarse), TPB, 0, s>>>(S.nCoarse, C.posCell.p, S.cellStart.p, cnt.p);
    S.rStartP.alloc(S.nCoarse + 1, s);
    exclusiveScan(cnt.p, S.rStartP.p, S.nCoarse, s);
    S.rListP.alloc(S.nFine, s);
    kStepLists<<<grid(S.nCoarse), TPB, 0, s>>>(S.nCoarse, C.posCell.p, S.cellStart.p, S.cellList.p, F.posOf.p,
                                               S.rStartP.p, S.rListP.p);
    S.prolongP.alloc(S.nFine, s);
    kProlongMap<<<grid(S.nFine), TPB, 0, s>>>(S.nFine, F.posCell.p, S.restrictAddr.p, C.posOf.p, S.prolongP.p);
    B2G_LAUNCH_CHECK();
    if (i == 0 && F.nEllEnt > 0)
    {
        GsSchedule& G = M.lev[0].gs;
        G.ellColCoarse.alloc(static_cast<size_t>(G.nEllEnt), s);
        kEllColCoarse<<<static_cast<unsigned>(std::min<long long>((G.nEllEnt + TPB - 1) / TPB, 65535LL)), TPB, 0, s>>>(
            G.nEllEnt, G.ellCol.p, S.prolongP.p, G.ellColCoarse.p);
        B2G_LAUNCH_CHECK();
    }
}

cudaMemPool_t libraryPool()
{
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    B2G_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) fail(B2G_ERR_STATE, "b2g: device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[dev])
    {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        B2G_CUDA(cudaMemPoolCreate(&pools[dev], &props));
        unsigned long long keep = ~0ULL;  // the attribute is a 64-bit unsigned integer
        B2G_CUDA(cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep));
    }
    return pools[dev];
}

const DeviceInfo& DeviceInfo::get()
{
    static DeviceInfo info = [] {
        DeviceInfo d;
        cudaGetDevice(&d.device);
        cudaDeviceGetAttribute(&d.numSMs, cudaDevAttrMultiProcessorCount, d.device);
        cudaDeviceGetAttribute(&d.maxSmemPerBlockOptin, cudaDevAttrMaxSharedMemoryPerBlockOptin, d.device);
        return d;
    }();
    return info;
}

}  // namespace b2g
