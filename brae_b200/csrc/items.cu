// items.cu -- the item schedule of a level: the multi-part exact Gauss-Seidel sweep (gs_kernels.cuh)
// running SEVERAL sweeps of one smoothing call in one launch, pipelined as pipe_kernels.cuh explains
// (sweep s+1 starts on a cell once every value its row reads is final; the combined steps T_s(c)).
//
// The sweep kernel is the same; what changes is what its "positions" are. Here they index ITEMS, the
// (sweep, cell) pairs, ordered by (part, step, sweep, position): each part walks its items step by
// step, a chunk holds items of one step, and the part publishes its progress in steps. Its window
// holds the results of the part's most recent items, a row's entry codes naming the item that
// produced the value it reads when that item is recent enough, else a gather from psi. The producer
// of an entry is the lower neighbour's item of the same sweep, or the upper neighbour's item of the
// previous sweep; in the first sweep an upper neighbour's value is the smoothing call's starting psi,
// which is gathered without a wait (it is overwritten only after this item is done).
//
// WHY A GATHER FROM psi READS THE RIGHT VERSION. psi holds one value per cell, overwritten by each
// sweep. A later version of the value an item reads is written by a later item of the same cell, and
// that item depends on this one by the recurrence (it reads this item's cell or is read by it), so it
// runs only after this item -- which gathers its values before it computes -- is done.
//
// FORWARD PROGRESS. A part now also waits for parts AFTER it (an upper neighbour's previous-sweep
// value), so every part must be resident at once: the launch is cooperative (all CTAs co-resident, or
// the launch fails), P <= the SM count at one CTA per SM. Waits are bounded as in every sweep.
//
// Reference: gaussSeidelSweeps, src/OpenFOAM/matrices/smooth_solver_cpp.cu:87-166, once per sweep.

#include "gs_kernels.cuh"
#include "hierarchy.cuh"

#include <algorithm>
#include <vector>

namespace b2g {
namespace {

constexpr int TPB = 256;
inline int grid(long long n) { return std::max(1, ceilDiv(n, TPB)); }

// What the classification kernels read about the items.
struct ItemView
{
    int n;                                   // cells
    const int* __restrict__ itemCell;        // [nItems]
    const unsigned char* __restrict__ itemSweep;
    const int* __restrict__ itemOf;          // [S][n] the item of (sweep, cell)
    const int* __restrict__ itemT;           // [nItems] its step
    const int* __restrict__ partOf;          // [n] by cell
    const int* __restrict__ chunkOf;         // [nItems]
    const int* __restrict__ chunkStart;      // [nChunks + 1]
    const int* __restrict__ posOf;           // [n] storage position of each cell
    const int* __restrict__ rowStart;        // [n + 1] by cell, the reference's row order
    const int* __restrict__ losortStart;     // [n + 1] (lower-side entries first in each row)
    const int* __restrict__ col;
    const int* __restrict__ entFace;
    int behind;

    // the item whose result an entry of (sweep s, cell c) reads: the lower neighbour's of sweep s, the
    // upper neighbour's of sweep s-1, none (the starting psi) for an upper neighbour in sweep 0
    __device__ int producer(int s, int o, bool lowerSide) const
    {
        if (lowerSide) return itemOf[static_cast<size_t>(s) * n + o];
        return s > 0 ? itemOf[static_cast<size_t>(s - 1) * n + o] : -1;
    }
    // a window read: produced by this part recently enough that the window still holds it when the
    // chunk reads (at most `behind` items before the chunk's end)
    __device__ bool window(int prod, bool same, int ch) const
    {
        return prod >= 0 && same && prod >= chunkStart[ch + 1] - behind;
    }
};

__global__ void kItemChunkOf(int nItems, int nChunks, const int* __restrict__ chunkStart, int* __restrict__ chunkOf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nItems) return;
    int lo = 0, hi = nChunks - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (chunkStart[mid] <= i) lo = mid; else hi = mid - 1;
    }
    chunkOf[i] = lo;
}

// pass 1: per item the gathers of values final as they are (the starting psi) and of values
// produced by items (with the waits they need: this part's producers outside the window wait for
// their chunk, other parts' for their progress), and the parts each part waits for
__global__ void kItemGatherCounts(int nItems, ItemView v, int* __restrict__ cntOld, int* __restrict__ cntNew,
                                  int* __restrict__ chunkNeedUp, int* __restrict__ chunkSameWait,
                                  unsigned* __restrict__ upBits, int words)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nItems) return;
    const int c = v.itemCell[i];
    const int s = v.itemSweep[i];
    const int p = v.partOf[c];
    const int ch = v.chunkOf[i];
    const int rb = v.rowStart[c];
    const int nLower = v.losortStart[c + 1] - v.losortStart[c];
    int gOld = 0, gNew = 0;
    for (int e = rb; e < v.rowStart[c + 1]; ++e)
    {
        const int o = v.col[e];
        const int prod = v.producer(s, o, e - rb < nLower);
        const bool same = v.partOf[o] == p;
        if (v.window(prod, same, ch)) continue;
        if (prod < 0)
        {
            ++gOld;
            continue;
        }
        ++gNew;
        if (same)
            atomicMax(&chunkSameWait[ch], v.chunkOf[prod]);
        else
        {
            atomicMax(&chunkNeedUp[ch], v.itemT[prod]);
            const int po = v.partOf[o];
            atomicOr(&upBits[static_cast<size_t>(p) * words + (po >> 5)], 1u << (po & 31));
        }
    }
    cntOld[i] = gOld;
    cntNew[i] = gNew;
}

// pass 2: the sliced-ELL codes and faces and the gather lists (a chunk's old values first, then the
// produced ones), the gather sources being storage positions in psi
__global__ void kItemSweepEntries(int nItems, ItemView v, int maxGat, const int* __restrict__ partChunkStart,
                                  const unsigned* __restrict__ itemEnt, const long long* __restrict__ chunkEnt0,
                                  const int* __restrict__ oldOff, const int* __restrict__ newOff,
                                  unsigned short* __restrict__ code, int* __restrict__ face, int* __restrict__ gatSrc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nItems) return;
    const int c = v.itemCell[i];
    const int s = v.itemSweep[i];
    const int p = v.partOf[c];
    const int ch = v.chunkOf[i];
    const int rb = v.rowStart[c];
    const int nLower = v.losortStart[c + 1] - v.losortStart[c];
    const long long ell = chunkEnt0[ch] + static_cast<long long>(itemEnt[i] & 0xffffffu);
    const int stage = (ch - partChunkStart[p]) % k::kStages;
    const int cs = v.chunkStart[ch];
    const int ce = v.chunkStart[ch + 1];
    const int base = oldOff[cs] + newOff[cs];
    const int g0 = base - (k::kWin + stage * maxGat);
    int gOld = base + (oldOff[i] - oldOff[cs]);
    int gNew = base + (oldOff[ce] - oldOff[cs]) + (newOff[i] - newOff[cs]);
    for (int e = rb; e < v.rowStart[c + 1]; ++e)
    {
        const int q = e - rb;
        const int o = v.col[e];
        const int prod = v.producer(s, o, q < nLower);
        const bool same = v.partOf[o] == p;
        unsigned short cd;
        if (v.window(prod, same, ch)) cd = static_cast<unsigned short>(prod & (k::kWin - 1));
        else
        {
            int& g = prod < 0 ? gOld : gNew;
            cd = static_cast<unsigned short>(g - g0);
            gatSrc[g++] = v.posOf[o];
        }
        code[ell + 32LL * q] = cd;
        face[ell + 32LL * q] = v.entFace[e];
    }
}

__global__ void kItemChunkRecs(int nCh, const int* __restrict__ chunkStart, const long long* __restrict__ chunkEnt0,
                               const int* __restrict__ chunkStep, const int* __restrict__ chunkNewStep,
                               const int* __restrict__ oldOff, const int* __restrict__ newOff,
                               const int* __restrict__ chunkNeedUp, const int* __restrict__ chunkSameWait,
                               const int2* __restrict__ chunkBlob, int* __restrict__ rec)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nCh) return;
    const int p0 = chunkStart[c];
    const int p1 = chunkStart[c + 1];
    int* r = rec + 12 * static_cast<size_t>(c);
    const int nOld = oldOff[p1] - oldOff[p0];
    r[0] = p0;
    r[1] = p1 - p0;
    r[2] = static_cast<int>(chunkEnt0[c]);
    r[3] = static_cast<int>(chunkEnt0[c + 1] - chunkEnt0[c]);
    r[4] = oldOff[p0] + newOff[p0];
    r[5] = nOld + newOff[p1] - newOff[p0];
    r[6] = chunkStep[c];
    r[7] = chunkNeedUp[c];
    r[8] = chunkSameWait[c];
    r[9] = chunkNewStep[c] | (nOld << 1);
    r[10] = chunkBlob[c].x;
    r[11] = chunkBlob[c].y;
}

__global__ void kItemFillShort(unsigned short* v, long long n, unsigned short value)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[i] = value;
}

__global__ void kItemFillInt(int* v, long long n, int value)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[i] = value;
}

}  // namespace

// The item schedule of L for S sweeps (see the head of this file), or null when it cannot be built
// (one part, or a level beyond the schedule's 32-bit item and entry counts).
std::unique_ptr<GsSchedule> buildGsItems(const LevelAddr& L, int S, cudaStream_t s)
{
    const GsSchedule& B = L.gs;
    const int n = L.nCells;
    const int P = B.nParts;
    if (S < 2 || n == 0 || P < 2) return nullptr;
    const long long nItemsLL = static_cast<long long>(S) * n;
    if (nItemsLL >= (1LL << 30) || 2LL * L.nFaces * S >= (1LL << 31)) return nullptr;
    const int nItems = static_cast<int>(nItemsLL);

    // ---- host: combined steps, items in (part, step, sweep, position) order ----
    const std::vector<int> depth = B.depth.download(s);
    const std::vector<int> lower = L.lower.download(s);
    const std::vector<int> upper = L.upper.download(s);
    const std::vector<int> posCell = B.posCell.download(s);
    const std::vector<int> partPos = B.partPosStart.download(s);  // parts are cell ranges
    const std::vector<int> rowStartH = L.rowStart.download(s);
    const int nF = L.nFaces;
    std::vector<int> T(static_cast<size_t>(nItems));
    std::copy(depth.begin(), depth.begin() + n, T.begin());
    for (int q = 1; q < S; ++q)
    {
        const int* prev = T.data() + static_cast<size_t>(q - 1) * n;
        int* cur = T.data() + static_cast<size_t>(q) * n;
        for (int c = 0; c < n; ++c) cur[c] = prev[c] + 1;
        for (int f = 0; f < nF; ++f) cur[lower[f]] = std::max(cur[lower[f]], prev[upper[f]] + 1);
        for (int f = 0; f < nF; ++f) cur[upper[f]] = std::max(cur[upper[f]], cur[lower[f]] + 1);
    }
    const int nSteps = *std::max_element(T.begin(), T.end()) + 1;
    std::vector<int> partOf(n);
    for (int p = 0; p < P; ++p)
        for (int c = partPos[p]; c < partPos[p + 1]; ++c) partOf[c] = p;
    // counting sort on (part, step); within a bucket items arrive by (sweep, position)
    const long long nBuckets = static_cast<long long>(P) * nSteps;
    if (nBuckets >= (1LL << 31)) return nullptr;
    std::vector<int> bucket(static_cast<size_t>(nBuckets) + 1, 0);
    for (int q = 0; q < S; ++q)
        for (int c = 0; c < n; ++c)
            ++bucket[static_cast<size_t>(partOf[c]) * nSteps + T[static_cast<size_t>(q) * n + c] + 1];
    for (size_t b = 1; b < bucket.size(); ++b) bucket[b] += bucket[b - 1];
    std::vector<int> itemCell(nItems), itemT(nItems), itemStore(nItems), itemOf(nItems);
    std::vector<unsigned char> itemSweep(nItems);
    {
        std::vector<int> cursor(bucket.begin(), bucket.end() - 1);
        for (int q = 0; q < S; ++q)
            for (int p = 0; p < n; ++p)
            {
                const int c = posCell[p];
                const int t = T[static_cast<size_t>(q) * n + c];
                const int at = cursor[static_cast<size_t>(partOf[c]) * nSteps + t]++;
                itemCell[at] = c;
                itemT[at] = t;
                itemStore[at] = p;
                itemSweep[at] = static_cast<unsigned char>(q);
                itemOf[static_cast<size_t>(q) * n + c] = at;
            }
    }
    std::vector<int>().swap(T);
    // groups: the non-empty (part, step) buckets
    std::vector<int> gStart, gStep, gPart;
    for (int p = 0; p < P; ++p)
        for (int t = 0; t < nSteps; ++t)
        {
            const size_t b = static_cast<size_t>(p) * nSteps + t;
            if (bucket[b + 1] > bucket[b])
            {
                gStart.push_back(bucket[b]);
                gStep.push_back(t);
                gPart.push_back(p);
            }
        }
    std::vector<int>().swap(bucket);
    const int nGroups = static_cast<int>(gStart.size());
    gStart.push_back(nItems);
    int maxGroup = 0, maxRow = 0;
    for (int g = 0; g < nGroups; ++g) maxGroup = std::max(maxGroup, gStart[g + 1] - gStart[g]);
    for (int c = 0; c < n; ++c) maxRow = std::max(maxRow, rowStartH[c + 1] - rowStartH[c]);
    if (maxRow > 255) return nullptr;
    const long long nnz = rowStartH[n];
    const int rowCap = std::max(1, std::min(maxRow, static_cast<int>((5LL * nnz + 4LL * n - 1) / (4LL * n))));
    const size_t smemCap = 200 * 1024;
    auto behindOf = [](int m) { return k::kWin - (k::kStages - 1) * m - 32; };
    auto fits = [&](int m, int e, int g) {
        return k::gsSmemBytes<double>(m, e, g, 1) <= smemCap && behindOf(m) >= m &&
               k::kWin + k::kStages * g + 1 <= k::kMaxTable;
    };

    // ---- device copies of what classification reads ----
    DBuf<int> dItemCell, dItemT, dItemOf, dPartOf, dChunkOf;
    DBuf<unsigned char> dItemSweep;
    dItemCell.upload(itemCell.data(), itemCell.size(), s);
    dItemT.upload(itemT.data(), itemT.size(), s);
    dItemOf.upload(itemOf.data(), itemOf.size(), s);
    dItemSweep.upload(itemSweep.data(), itemSweep.size(), s);
    dPartOf.upload(partOf.data(), partOf.size(), s);
    dChunkOf.alloc(nItems, s);
    auto G = std::make_unique<GsSchedule>();
    G->items = S;
    G->itemStore.upload(itemStore.data(), itemStore.size(), s);
    const int words = (P + 31) / 32;
    int M = std::min(k::kMaxCompute, std::max(32, ((maxGroup + 31) / 32) * 32));
    for (int attempt = 0;; ++attempt)
    {
        int E = ((std::max(M * rowCap, 32 * maxRow) + 31) / 32) * 32;
        while (M > 32 && !fits(M, E, M)) { M -= 32; E = ((std::max(M * rowCap, 32 * maxRow) + 31) / 32) * 32; }
        if (!fits(M, E, 32)) return nullptr;
        // host chunking: chunks of at most M items of one (part, step), grown slice by slice
        std::vector<int> hChunkStart, hChunkStep, hChunkNewStep, hPartChunk(P + 1, 0);
        std::vector<long long> hChunkEnt0;
        std::vector<unsigned> hItemEnt(static_cast<size_t>(nItems) + 8, 0u);
        long long ent = 0;
        int prevPart = -1;
        for (int g = 0; g < nGroups; ++g)
        {
            const int gs = gStart[g], ge = gStart[g + 1];
            int cs = gs;
            while (cs < ge)
            {
                int ce = cs;
                long long nEnt = 0;
                while (ce < ge && ce - cs < M)
                {
                    const int sEnd = std::min({ce + 32, ge, cs + M});
                    int w = 0;
                    for (int i = ce; i < sEnd; ++i)
                        w = std::max(w, rowStartH[itemCell[i] + 1] - rowStartH[itemCell[i]]);
                    if (nEnt + 32LL * w > E && ce > cs) break;
                    for (int i = ce; i < sEnd; ++i)
                        hItemEnt[i] = (static_cast<unsigned>(w) << 24) | static_cast<unsigned>(nEnt + (i - ce));
                    nEnt += 32LL * w;
                    ce = sEnd;
                }
                hChunkStart.push_back(cs);
                hChunkEnt0.push_back(ent);
                hChunkStep.push_back(gStep[g]);
                hChunkNewStep.push_back(cs == gs && prevPart == gPart[g] ? 1 : 0);
                hPartChunk[gPart[g] + 1]++;
                prevPart = gPart[g];
                ent += nEnt;
                cs = ce;
            }
        }
        const int nCh = static_cast<int>(hChunkStart.size());
        hChunkStart.push_back(nItems);
        hChunkEnt0.push_back(ent);
        for (int q = 0; q < P; ++q) hPartChunk[q + 1] += hPartChunk[q];
        if (ent >= (1LL << 31)) return nullptr;
        const int behind = behindOf(M);
        DBuf<int> chunkStart, chunkStep, chunkNewStep, chunkNeedUp, chunkSameWait, cntOld, cntNew, oldOff, newOff;
        DBuf<long long> chunkEnt0;
        chunkStart.upload(hChunkStart.data(), hChunkStart.size(), s);
        chunkStep.upload(hChunkStep.data(), hChunkStep.size(), s);
        chunkNewStep.upload(hChunkNewStep.data(), hChunkNewStep.size(), s);
        chunkEnt0.upload(hChunkEnt0.data(), hChunkEnt0.size(), s);
        G->posEnt.upload(hItemEnt.data(), hItemEnt.size(), s);
        chunkNeedUp.alloc(nCh, s);
        chunkSameWait.alloc(nCh, s);
        kItemFillInt<<<grid(nCh), TPB, 0, s>>>(chunkNeedUp.p, nCh, -1);
        kItemFillInt<<<grid(nCh), TPB, 0, s>>>(chunkSameWait.p, nCh, -1);
        kItemChunkOf<<<grid(nItems), TPB, 0, s>>>(nItems, nCh, chunkStart.p, dChunkOf.p);
        B2G_LAUNCH_CHECK();
        DBuf<unsigned> upBits;
        upBits.alloc(static_cast<size_t>(P) * words, s);
        upBits.zero(s);
        ItemView v;
        v.n = n;
        v.itemCell = dItemCell.p;
        v.itemSweep = dItemSweep.p;
        v.itemOf = dItemOf.p;
        v.itemT = dItemT.p;
        v.partOf = dPartOf.p;
        v.chunkOf = dChunkOf.p;
        v.chunkStart = chunkStart.p;
        v.posOf = B.posOf.p;
        v.rowStart = L.rowStart.p;
        v.losortStart = L.losortStart.p;
        v.col = L.col.p;
        v.entFace = L.entFace.p;
        v.behind = behind;
        cntOld.alloc(nItems, s);
        cntNew.alloc(nItems, s);
        kItemGatherCounts<<<grid(nItems), TPB, 0, s>>>(nItems, v, cntOld.p, cntNew.p, chunkNeedUp.p, chunkSameWait.p,
                                                        upBits.p, words);
        B2G_LAUNCH_CHECK();
        oldOff.alloc(static_cast<size_t>(nItems) + 1, s);
        newOff.alloc(static_cast<size_t>(nItems) + 1, s);
        const long long nGather = exclusiveScan(cntOld.p, oldOff.p, nItems, s) + exclusiveScan(cntNew.p, newOff.p, nItems, s);
        if (nGather >= (1LL << 31)) return nullptr;
        const std::vector<int> hOldOff = oldOff.download(s);
        const std::vector<int> hNewOff = newOff.download(s);
        int maxGat = 0;
        for (int c = 0; c < nCh; ++c)
            maxGat = std::max(maxGat, hOldOff[hChunkStart[c + 1]] - hOldOff[hChunkStart[c]] +
                                          hNewOff[hChunkStart[c + 1]] - hNewOff[hChunkStart[c]]);
        maxGat = ((maxGat + 1) / 2) * 2;
        if (!fits(M, E, maxGat) && M > 32 && attempt < 16)
        {
            M -= 32;
            continue;
        }
        if (!fits(M, E, maxGat)) return nullptr;
        G->nParts = P;
        G->maxDepth = nSteps - 1;
        G->nChunks = nCh;
        G->maxCells = M;
        G->maxEnt = E;
        G->maxGat = maxGat;
        G->ahead = 0;
        G->behind = behind;
        G->nEll = ent;
        G->nGather = nGather;
        G->nPadded = ((nItems + k::kFill - 1) / k::kFill) * k::kFill;
        G->nAlloc = G->nPadded + k::kFill;
        G->partChunkStart.upload(hPartChunk.data(), hPartChunk.size(), s);
        G->gsCode.alloc(std::max<long long>(ent, 1), s);
        G->gsEntFace.alloc(std::max<long long>(ent, 1), s);
        G->gatSrc.alloc(std::max<long long>(nGather, 1) + 8, s);
        if (ent)
        {
            kItemFillShort<<<std::min<long long>(ceilDiv(ent, TPB), 8192), TPB, 0, s>>>(
                G->gsCode.p, ent, static_cast<unsigned short>(k::kWin + k::kStages * maxGat));
            kItemFillInt<<<std::min<long long>(ceilDiv(ent, TPB), 8192), TPB, 0, s>>>(G->gsEntFace.p, ent, -1);
        }
        kItemSweepEntries<<<grid(nItems), TPB, 0, s>>>(nItems, v, maxGat, G->partChunkStart.p, G->posEnt.p,
                                                        chunkEnt0.p, oldOff.p, newOff.p, G->gsCode.p, G->gsEntFace.p,
                                                        G->gatSrc.p);
        B2G_LAUNCH_CHECK();
        std::vector<int2> hBlob(nCh);
        long long b64 = 0, b32 = 0;
        for (int c = 0; c < nCh; ++c)
        {
            const int m = hChunkStart[c + 1] - hChunkStart[c];
            const int ne = static_cast<int>(hChunkEnt0[c + 1] - hChunkEnt0[c]);
            hBlob[c] = make_int2(static_cast<int>(b64 / 16), static_cast<int>(b32 / 16));
            b64 += k::blobLayout<double>(m, ne, 1).bytes;
            b32 += k::blobLayout<float>(m, ne, 1).bytes;
        }
        if (b64 / 16 >= (1LL << 31)) return nullptr;
        G->blobBytes64 = b64;
        G->blobBytes32 = b32;
        DBuf<int2> chunkBlob;
        chunkBlob.upload(hBlob.data(), hBlob.size(), s);
        G->chunkRec.alloc(12 * static_cast<size_t>(nCh), s);
        kItemChunkRecs<<<grid(nCh), TPB, 0, s>>>(nCh, chunkStart.p, chunkEnt0.p, chunkStep.p, chunkNewStep.p, oldOff.p,
                                                  newOff.p, chunkNeedUp.p, chunkSameWait.p, chunkBlob.p, G->chunkRec.p);
        B2G_LAUNCH_CHECK();
        // the parts each part waits for, and which parts others wait for
        const std::vector<unsigned> hUp = upBits.download(s);
        std::vector<int> upStart(P + 1, 0), upList;
        for (int q = 0; q < P; ++q)
        {
            upStart[q] = static_cast<int>(upList.size());
            for (int r = 0; r < P; ++r)
                if (hUp[static_cast<size_t>(q) * words + (r >> 5)] & (1u << (r & 31))) upList.push_back(r);
        }
        upStart[P] = static_cast<int>(upList.size());
        std::vector<int> hasDown(P, 0);
        for (int r : upList) hasDown[r] = 1;
        G->hasDown.upload(hasDown.data(), hasDown.size(), s);
        G->upStart.upload(upStart.data(), upStart.size(), s);
        if (upList.empty()) upList.push_back(0);
        G->upList.upload(upList.data(), upList.size(), s);
        // the parts' item ranges (the window fill bookkeeping reads them; an item schedule fills nothing)
        std::vector<int> partItem(P + 1, 0);
        for (int q = 0; q < P; ++q) partItem[q + 1] = hChunkStart[hPartChunk[q + 1]];
        G->partPosStart.upload(partItem.data(), partItem.size(), s);
        B2G_CUDA(cudaStreamSynchronize(s));
        break;
    }
    G->progress.alloc(static_cast<size_t>(P + 1) * k::kProgressStride, s);
    G->progress.zero(s);
    B2G_CUDA(cudaStreamSynchronize(s));
    return G;
}

}  // namespace b2g
