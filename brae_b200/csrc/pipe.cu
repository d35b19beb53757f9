// pipe.cu -- the pipelined multi-sweep Gauss-Seidel launch (pipe_kernels.cuh): its schedule, built
// once per (level, sweep count, shape) on the host from the level's addressing, and the choice, by
// measurement on the device, between its shapes (one CTA; a cluster of 2..16 CTAs; the grid form on
// 148 or 74 resident CTAs), the item schedule (items.cu) and the sweep-by-sweep launches. The same
// launch also runs the multicolour FP32 smoother's calls, with the colours as its steps
// (colourSchedule, Matrix::ensureMcPipe).
//
// Reference: the sweeps it reproduces are gaussSeidelSweeps, src/OpenFOAM/matrices/
// smooth_solver_cpp.cu:87-166 (forward only for GaussSeidel, :144), called nSweeps times per
// smoothing call by GaussSeidelSmoother::smooth (gamg_solver_cpp.cu:234-317).

#include "pipe_kernels.cuh"
#include "solver.cuh"

#include <algorithm>
#include <atomic>
#include <vector>

namespace b2g {
namespace {

constexpr size_t kPipeSmemCap = 220 * 1024;  // dynamic shared memory of one rank: its psi slots and step table

// The level's addressing on the host, as the schedule builder reads it.
struct LevelHost
{
    int n = 0, nF = 0;
    std::vector<int> lower, upper, depth, posCell, posRow, entColPos;
};

LevelHost download(const LevelAddr& L, cudaStream_t s)
{
    LevelHost H;
    H.n = L.nCells;
    H.nF = L.nFaces;
    H.lower = L.lower.download(s);
    H.upper = L.upper.download(s);
    H.depth = L.gs.depth.download(s);
    H.posCell = L.gs.posCell.download(s);
    H.posRow = L.gs.posRow.download(s);
    H.entColPos = L.gs.entColPos.download(s);
    H.lower.resize(H.nF);
    H.upper.resize(H.nF);
    H.posRow.resize(static_cast<size_t>(H.n) + 1);
    H.entColPos.resize(2 * static_cast<size_t>(H.nF));
    return H;
}

// T_s(c) of every item (s, c), s < S (pipe_kernels.cuh): T_0 is the depth; then per sweep the upper
// neighbours' and the cell's own previous step, then the lower neighbours' in face order (faces are
// sorted by owner, so a face's owner has its final value when the face is reached).
std::vector<int> combinedSteps(const LevelHost& H, int S, int& nSteps)
{
    const size_t n = static_cast<size_t>(H.n);
    std::vector<int> T(static_cast<size_t>(S) * n);
    std::copy(H.depth.begin(), H.depth.begin() + n, T.begin());
    for (int s = 1; s < S; ++s)
    {
        const int* prev = T.data() + (s - 1) * n;
        int* cur = T.data() + s * n;
        for (size_t c = 0; c < n; ++c) cur[c] = prev[c] + 1;
        for (int f = 0; f < H.nF; ++f) cur[H.lower[f]] = std::max(cur[H.lower[f]], prev[H.upper[f]] + 1);
        for (int f = 0; f < H.nF; ++f) cur[H.upper[f]] = std::max(cur[H.upper[f]], cur[H.lower[f]] + 1);
    }
    nSteps = T.empty() ? 0 : *std::max_element(T.begin(), T.end()) + 1;
    return T;
}

// The schedule for R ranks, or null when a rank's slots do not fit the shared memory (the grid form:
// R resident CTAs, psi in global memory, each rank's neighbour ranks listed).
std::unique_ptr<PipeSchedule> assemble(const LevelHost& H, const std::vector<int>& T, int S, int nSteps, int R,
                                       size_t valueBytes, cudaStream_t s, bool grid = false)
{
    const int n = H.n;
    if (n == 0 || R < 1 || (!grid && R > k::kPipeMaxRanks)) return nullptr;
    // ranks: contiguous cell ranges; slots: a rank's cells in position order
    std::vector<int> rankOf(n), slotOf(n), count(R, 0);
    for (int c = 0; c < n; ++c) rankOf[c] = static_cast<int>(static_cast<long long>(c) * R / n);
    for (int p = 0; p < n; ++p)
    {
        const int c = H.posCell[p];
        slotOf[c] = count[rankOf[c]]++;
    }
    const int maxLocal = grid ? 0 : *std::max_element(count.begin(), count.end());
    if (maxLocal >= (1 << 24)) return nullptr;
    if (!grid && k::pipeStepTableAt(maxLocal, valueBytes) + sizeof(int) * (static_cast<size_t>(nSteps) + 1) > kPipeSmemCap)
        return nullptr;
    std::vector<int> localPos(std::max<size_t>(static_cast<size_t>(R) * maxLocal, 1), 0);
    if (!grid)
        for (int p = 0; p < n; ++p)
        {
            const int c = H.posCell[p];
            localPos[static_cast<size_t>(rankOf[c]) * maxLocal + slotOf[c]] = p;
        }
    if (grid && sizeof(int) * (nSteps + 1) > 48 * 1024) return nullptr;
    // the grid form: a value is named by its position, and a row's value slot is its position
    if (grid)
        for (int p = 0; p < n; ++p) slotOf[H.posCell[p]] = p;
    // items, rank-major then by step, in position order within a (rank, step)
    const size_t stride = static_cast<size_t>(nSteps) + 1;
    std::vector<int> start(static_cast<size_t>(R) * stride + 1, 0);
    for (int c = 0; c < n; ++c)
        for (int q = 0; q < S; ++q) ++start[static_cast<size_t>(rankOf[c]) * stride + T[static_cast<size_t>(q) * n + c] + 1];
    for (size_t i = 1; i < start.size(); ++i) start[i] += start[i - 1];
    std::vector<int> cursor(start.begin(), start.end() - 1);
    std::vector<int4> item(static_cast<size_t>(S) * n);
    for (int p = 0; p < n; ++p)
    {
        const int c = H.posCell[p];
        for (int q = 0; q < S; ++q)
        {
            const int at = cursor[static_cast<size_t>(rankOf[c]) * stride + T[static_cast<size_t>(q) * n + c]]++;
            item[at] = make_int4(p, slotOf[c], H.posRow[p], H.posRow[p + 1]);
        }
    }
    // per rank and step its item range [stepStart[r][t], stepStart[r][t + 1]): the last entry of a
    // rank's row is the first of the next rank's, so the table is start[] read per rank
    std::vector<int> stepStart(static_cast<size_t>(R) * stride);
    for (int r = 0; r < R; ++r)
        for (size_t t = 0; t < stride; ++t) stepStart[r * stride + t] = start[r * stride + t];
    std::vector<unsigned> entAddr;
    if (!grid)
    {
        entAddr.resize(H.entColPos.size());
        for (size_t e = 0; e < entAddr.size(); ++e)
        {
            const int c = H.posCell[H.entColPos[e]];
            entAddr[e] = static_cast<unsigned>(rankOf[c]) << 24 | static_cast<unsigned>(slotOf[c]);
        }
    }
    auto P = std::make_unique<PipeSchedule>();
    P->sweeps = S;
    P->ranks = R;
    P->nSteps = nSteps;
    P->maxLocal = maxLocal;
    P->stepStart.upload(stepStart.data(), stepStart.size(), s);
    P->item.upload(item.data(), item.size(), s);
    if (!grid) P->entAddr.upload(entAddr.data(), std::max<size_t>(entAddr.size(), 1), s);
    P->localPos.upload(localPos.data(), localPos.size(), s);
    P->localCount.upload(count.data(), count.size(), s);
    if (grid)
    {
        // each rank's neighbour ranks: the other ends of its cells' faces
        std::vector<std::vector<int>> nb(R);
        for (int f = 0; f < H.nF; ++f)
        {
            const int a = rankOf[H.lower[f]], b = rankOf[H.upper[f]];
            if (a == b) continue;
            nb[a].push_back(b);
            nb[b].push_back(a);
        }
        std::vector<int> nbrStart(static_cast<size_t>(R) + 1, 0), nbrList;
        for (int r = 0; r < R; ++r)
        {
            std::sort(nb[r].begin(), nb[r].end());
            nb[r].erase(std::unique(nb[r].begin(), nb[r].end()), nb[r].end());
            nbrList.insert(nbrList.end(), nb[r].begin(), nb[r].end());
            nbrStart[r + 1] = static_cast<int>(nbrList.size());
        }
        P->grid = true;
        P->nbrStart.upload(nbrStart.data(), nbrStart.size(), s);
        P->nbrList.upload(nbrList.data(), std::max<size_t>(nbrList.size(), 1), s);
        P->progress.alloc(static_cast<size_t>(R) * k::kProgressStride, s);
    }
    B2G_CUDA(cudaStreamSynchronize(s));  // the host vectors go out of scope
    return P;
}

// The multicolour smoother's sweeps as a pipelined schedule: item (sweep s, cell c) runs at step
// s * stepsPerSweep + k for a cell of colour k; symmetric sweeps visit the colours forward then back,
// each cell twice a sweep. No two cells of a colour share a face, so a step's items are independent,
// and each row reads the values the colour-by-colour sweep gives it. Null when a cell has no colour.
std::unique_ptr<PipeSchedule> colourSchedule(const LevelHost& H, const Colouring& C, const std::vector<int>& rowPos,
                                             int nSweeps, bool symmetric, int R, cudaStream_t s)
{
    const int n = H.n;
    std::vector<int> colourOf(n, -1);
    for (int k = 0; k < C.nColours; ++k)
        for (int r = C.colourStart[k]; r < C.colourStart[k + 1]; ++r)
            if (rowPos[r] >= 0) colourOf[H.posCell[rowPos[r]]] = k;
    for (int c = 0; c < n; ++c)
        if (colourOf[c] < 0) return nullptr;
    const int per = symmetric ? 2 : 1;
    const int stepsPerSweep = per * C.nColours;
    const int S = nSweeps * per;
    std::vector<int> T(static_cast<size_t>(S) * n);
    for (int sw = 0; sw < nSweeps; ++sw)
        for (int c = 0; c < n; ++c)
        {
            const int k = colourOf[c];
            T[static_cast<size_t>(sw * per) * n + c] = sw * stepsPerSweep + k;
            if (symmetric) T[static_cast<size_t>(sw * per + 1) * n + c] = sw * stepsPerSweep + 2 * C.nColours - 1 - k;
        }
    return assemble(H, T, S, nSweeps * stepsPerSweep, R, sizeof(float), s);
}

template <class T>
void allowPipeSmem()
{
    static std::atomic<unsigned long long> done{0};  // one bit per device
    int dev = 0;
    B2G_CUDA(cudaGetDevice(&dev));
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load() & bit) return;
    B2G_CUDA(cudaFuncSetAttribute(k::gsPipe<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(kPipeSmemCap)));
    B2G_CUDA(cudaFuncSetAttribute(k::gsPipe<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(kPipeSmemCap)));
    // clusters above 8 CTAs are non-portable: opt in (refused on devices without them; the tuner
    // then finds no such shape resident)
    if (cudaFuncSetAttribute(k::gsPipe<T, true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
        cudaGetLastError();
    if constexpr (sizeof(T) == 4)
    {
        // the multicolour smoother's launches (the colours as steps)
        B2G_CUDA(cudaFuncSetAttribute(k::gsPipe<T, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kPipeSmemCap)));
        B2G_CUDA(cudaFuncSetAttribute(k::gsPipe<T, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kPipeSmemCap)));
        if (cudaFuncSetAttribute(k::gsPipe<T, true, true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess)
            cudaGetLastError();
    }
    done.fetch_or(bit);
}

// The launch configuration of a pipelined call.
struct PipeLaunch
{
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg;
    PipeLaunch(int ranks, size_t smem, cudaStream_t s)
    {
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = static_cast<unsigned>(ranks);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg = cudaLaunchConfig_t{};
        cfg.gridDim = dim3(static_cast<unsigned>(ranks));
        cfg.blockDim = dim3(k::kPipeBlock);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
};

template <class T>
bool pipeClusterFits(int ranks, size_t smem, cudaStream_t s, bool fma = false)
{
    PipeLaunch L(ranks, smem, s);
    int n = 0;
    cudaError_t e;
    if constexpr (sizeof(T) == 4)
        e = fma ? cudaOccupancyMaxActiveClusters(&n, k::gsPipe<T, true, true>, &L.cfg)
                : cudaOccupancyMaxActiveClusters(&n, k::gsPipe<T, true>, &L.cfg);
    else
        e = cudaOccupancyMaxActiveClusters(&n, k::gsPipe<T, true>, &L.cfg);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        return false;
    }
    return n >= 1;
}

// Whether `ranks` CTAs of the grid form can all be resident (its launch is cooperative).
template <class T>
bool pipeGridFits(int ranks, size_t smem)
{
    if (smem > 48 * 1024) return false;
    int dev = 0, sms = 0, perSm = 0;
    B2G_CUDA(cudaGetDevice(&dev));
    B2G_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k::gsPipeGrid<T>, k::kPipeGridBlock, smem) != cudaSuccess)
    {
        cudaGetLastError();
        return false;
    }
    return ranks <= perSm * sms;
}

int smCount()
{
    int dev = 0, sms = 0;
    B2G_CUDA(cudaGetDevice(&dev));
    B2G_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return sms;
}

int pipeKey(int sweeps, size_t valueBytes) { return sweeps * 16 + static_cast<int>(valueBytes); }

}  // namespace

size_t pipeSmemBytes(const PipeSchedule& P, size_t valueBytes)
{
    const size_t table = sizeof(int) * (static_cast<size_t>(P.nSteps) + 1);
    return P.grid ? table : k::pipeStepTableAt(P.maxLocal, valueBytes) + table;
}

template <class T>
k::PipeArgs<T> Matrix::pipeArgs(int level, const PipeSchedule& P, T* psiL, const T* src)
{
    k::PipeArgs<T> a;
    a.A = rowsOf(mesh->lev[level], data<T>().coef[level]);
    a.nSteps = P.nSteps;
    a.maxLocal = P.maxLocal;
    a.stepStart = P.stepStart.p;
    a.item = P.item.p;
    a.entAddr = P.entAddr.p;
    a.localPos = P.localPos.p;
    a.localCount = P.localCount.p;
    a.b = src;
    a.psi = psiL;
    return a;
}

template <class T>
void Matrix::pipeLaunch(int level, const PipeSchedule& P, T* psiL, const T* src, bool fma)
{
    const k::PipeArgs<T> a = pipeArgs<T>(level, P, psiL, src);
    const size_t smem = pipeSmemBytes(P, sizeof(T));
    if (P.grid)
    {
        k::PipeGridSync g;
        g.progress = P.progress.p;
        g.nbrStart = P.nbrStart.p;
        g.nbrList = P.nbrList.p;
        g.spinLimit = spinLimit;
        g.err = err.p;
        g.publish = publish;
        B2G_CUDA(cudaMemsetAsync(P.progress.p, 0, P.progress.bytes(), stream));
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(static_cast<unsigned>(P.ranks));
        cfg.blockDim = dim3(k::kPipeGridBlock);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = stream;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        B2G_CUDA(cudaLaunchKernelEx(&cfg, k::gsPipeGrid<T>, a, g));
        launches += 2;
        return;
    }
    if constexpr (sizeof(T) == 4)
        if (fma)
        {
            // the multicolour smoother's arithmetic
            if (P.ranks == 1)
            {
                k::gsPipe<T, false, true><<<1, k::kPipeBlock, smem, stream>>>(a);
                B2G_LAUNCH_CHECK();
            }
            else
            {
                PipeLaunch C(P.ranks, smem, stream);
                B2G_CUDA(cudaLaunchKernelEx(&C.cfg, k::gsPipe<T, true, true>, a));
            }
            ++launches;
            return;
        }
    if (fma) fail(B2G_ERR_STATE, "b2g: the multicolour pipelined launch is FP32 only");
    if (P.ranks == 1)
    {
        k::gsPipe<T, false><<<1, k::kPipeBlock, smem, stream>>>(a);
        B2G_LAUNCH_CHECK();
    }
    else
    {
        PipeLaunch C(P.ranks, smem, stream);
        B2G_CUDA(cudaLaunchKernelEx(&C.cfg, k::gsPipe<T, true>, a));
    }
    ++launches;
}

// An item schedule's buffers on this matrix, the chunk blobs refilled when the coefficients changed
// since they were filled (outside any capture).
template <class T>
typename VCycleData<T>::ItemBuffers& Matrix::itemBuffers(int level, const GsSchedule& G)
{
    VCycleData<T>& D = data<T>();
    auto& B = D.items[std::make_pair(level, G.items)];
    if (B.gen != coefGen)
    {
        if (capturing) fail(B2G_ERR_STATE, "b2g: an item schedule's blobs were not filled before the capture");
        // the blobs' padding is zeroed when the buffers are new; a refill writes the same bytes
        const long long bytes = sizeof(T) == 8 ? G.blobBytes64 : G.blobBytes32;
        const void* blobWas = B.blob.p;
        const size_t blobN = B.blob.n;
        B.blob.ensure(static_cast<size_t>(std::max<long long>(bytes, 16)), stream);
        if (B.blob.p != blobWas || B.blob.n != blobN) B.blob.zero(stream);
        const void* bWas = B.b.p;
        const size_t bN = B.b.n;
        B.b.ensure(static_cast<size_t>(std::max(G.nAlloc, 1)), stream);
        if (B.b.p != bWas || B.b.n != bN) B.b.zero(stream);
        if (G.nChunks)
            k::buildChunkBlobs<T><<<std::min(G.nChunks, 65535), 128, 0, stream>>>(
                G.nChunks, reinterpret_cast<const int4*>(G.chunkRec.p), D.coef[level].gsDiag.p, G.posEnt.p,
                G.gsCode.p, G.gsEntFace.p, v64.coef[level].upper.p, B.blob.p, G.itemStore.p);
        B2G_LAUNCH_CHECK();
        B.gen = coefGen;
    }
    return B;
}

namespace {
template <class T>
__global__ void kByItem(int nItems, const int* __restrict__ itemStore, const T* __restrict__ src, T* __restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nItems; i += gridDim.x * blockDim.x)
        out[i] = src[itemStore[i]];
}
}  // namespace

// The item schedule's sweeps in one launch: the source by item, then the multi-part sweep over the
// items, launched cooperatively (every part resident at once: parts wait for later parts too).
template <class T>
void Matrix::itemsLaunch(int level, const GsSchedule& G, T* psiL, const T* src)
{
    auto& B = itemBuffers<T>(level, G);
    const int nItems = G.items * mesh->lev[level].nCells;
    kByItem<T><<<std::min(ceilDiv(nItems, 256), 4096), 256, 0, stream>>>(nItems, G.itemStore.p, src, B.b.p);
    B2G_LAUNCH_CHECK();
    k::GsArgs<T> a;
    a.nParts = G.nParts;
    a.maxCells = G.maxCells;
    a.maxEnt = G.maxEnt;
    a.maxGat = G.maxGat;
    a.ahead = 0;
    a.nPadded = G.nPadded;
    a.partChunkStart = G.partChunkStart.p;
    a.partPosStart = G.partPosStart.p;
    a.chunkRec = reinterpret_cast<const int4*>(G.chunkRec.p);
    a.upStart = G.upStart.p;
    a.upList = G.upList.p;
    a.hasDown = G.hasDown.p;
    a.blob = B.blob.p;
    a.gatSrc = G.gatSrc.p;
    a.b = B.b.p;
    a.psi = psiL;
    a.progress = G.progress.p;
    a.ticket = reinterpret_cast<int*>(G.progress.p + static_cast<size_t>(G.nParts) * k::kProgressStride);
    a.items = 1;
    a.spinLimit = spinLimit;
    a.publish = publish;
    a.err = err.p;
    a.trace = nullptr;
    a.traceDepths = 0;
    B2G_CUDA(cudaMemsetAsync(G.progress.p, 0, G.progress.bytes(), stream));
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(G.nParts));
    cfg.blockDim = dim3(static_cast<unsigned>(G.maxCells + 128));
    cfg.dynamicSmemBytes = k::gsSmemBytes<T>(G.maxCells, G.maxEnt, G.maxGat, 1);
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    B2G_CUDA(cudaLaunchKernelEx(&cfg, k::gsSweep<T>, a));
    launches += 2;
}

// The pipelined smoothing call of `level` for nSweeps sweeps, tried once per (level, sweep count,
// value type) on this matrix's values: every shared-memory shape whose slots fit (one CTA; clusters
// of 2, 4, 8, 16 CTAs that can be resident) and, on a multi-part level, the item schedule, against
// the sweep-by-sweep launches; the fastest is kept. Every shape computes every row from the same
// operands in the same order, so the choice changes the time only. Outside any capture (it
// synchronises); the work vectors it sweeps are scratch.
template <class T>
void Matrix::ensurePipe(int level, int nSweeps)
{
    LevelAddr& L = mesh->lev[level];
    const int key = pipeKey(nSweeps, sizeof(T));
    if (L.pipe.count(key)) return;
    PipeChoice& C = L.pipe[key];
    if (nSweeps < 2 || L.nCells == 0) return;
    allowPipeSmem<T>();
    DBuf<T> x, b;
    x.alloc(nAlloc(level), stream);
    b.alloc(nAlloc(level), stream);
    x.zero(stream);
    b.zero(stream);
    cudaEvent_t e0, e1;
    B2G_CUDA(cudaEventCreate(&e0));
    B2G_CUDA(cudaEventCreate(&e1));
    const long long l0 = launches;
    auto timeIt = [&](auto&& launch) {
        launch();  // warm
        B2G_CUDA(cudaEventRecord(e0, stream));
        for (int i = 0; i < 3; ++i) launch();
        B2G_CUDA(cudaEventRecord(e1, stream));
        B2G_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        B2G_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms / 3.f;
    };
    // sweep by sweep: the resident block where the level takes it, else one launch per sweep
    C.msSweeps = timeIt([&] {
        if (!residentSweeps<T>(level, x.p, b.p, nSweeps))
            for (int sw = 0; sw < nSweeps; ++sw) gsLaunch<T>(L, data<T>().coef[level], x.p, b.p, nullptr, false);
    });
    checkDeviceError();
    float best = C.msSweeps;
    if (L.nCells <= k::kPipeMaxRanks * static_cast<int>(kPipeSmemCap / sizeof(T)))
    {
        const LevelHost H = download(L, stream);
        int nSteps = 0;
        const std::vector<int> Tsteps = combinedSteps(H, nSweeps, nSteps);
        for (int R : {1, 2, 4, 8, 16})
        {
            std::unique_ptr<PipeSchedule> P = assemble(H, Tsteps, nSweeps, nSteps, R, sizeof(T), stream);
            if (!P) continue;
            if (R > 1 && !pipeClusterFits<T>(R, pipeSmemBytes(*P, sizeof(T)), stream)) continue;
            const float ms = timeIt([&] { pipeLaunch<T>(level, *P, x.p, b.p); });
            if (C.msPipe == 0.f || ms < C.msPipe) C.msPipe = ms;
            if (ms < best)
            {
                best = ms;
                C.sched = std::move(P);
                C.mode = 1;
            }
        }
    }
    if (L.gs.nParts > 1)
    {
        // the grid form: one CTA per SM, or per two
        const LevelHost H = download(L, stream);
        int nSteps = 0;
        const std::vector<int> Tsteps = combinedSteps(H, nSweeps, nSteps);
        const int sms = smCount();
        for (int R : {sms, sms / 2})
        {
            if (R < 2 || R > L.nCells) continue;
            std::unique_ptr<PipeSchedule> P = assemble(H, Tsteps, nSweeps, nSteps, R, sizeof(T), stream, true);
            if (!P || !pipeGridFits<T>(R, pipeSmemBytes(*P, sizeof(T)))) continue;
            float ms = 0.f;
            try
            {
                ms = timeIt([&] { pipeLaunch<T>(level, *P, x.p, b.p); });
                checkDeviceError();
            }
            catch (const Error&)
            {
                // a cooperative launch of that many CTAs refused here
                cudaGetLastError();
                continue;
            }
            if (C.msGrid == 0.f || ms < C.msGrid) C.msGrid = ms;
            if (ms < best)
            {
                best = ms;
                C.sched = std::move(P);
                C.mode = 1;
            }
        }
        std::unique_ptr<GsSchedule> G = buildGsItems(L, nSweeps, stream);
        float ms = 0.f;
        if (G)
        {
            try
            {
                ms = timeIt([&] { itemsLaunch<T>(level, *G, x.p, b.p); });
                checkDeviceError();
            }
            catch (const Error&)
            {
                // a cooperative launch of that many parts refused here: no item schedule for the level
                cudaGetLastError();
                G.reset();
                data<T>().items.erase(std::make_pair(level, nSweeps));
            }
        }
        if (G)
        {
            C.msItems = ms;
            if (ms < best)
            {
                best = ms;
                C.items = std::move(G);
                C.sched.reset();
                C.mode = 2;
            }
            else
            {
                // not kept: this matrix's buffers for it go too
                data<T>().items.erase(std::make_pair(level, nSweeps));
            }
        }
    }
    launches = l0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    B2G_CUDA(cudaStreamSynchronize(stream));
}

// The multicolour smoothing call of nSweeps sweeps on `level` as one pipelined launch over the colours
// (colourSchedule), on one CTA or a cluster of 2-16, against the tuned colour-by-colour shape
// (Matrix::tuneMulticolour): the faster is kept. Both compute every row with the same fused
// multiply-adds in the same order on the same values, so the choice changes the time only.
void Matrix::ensureMcPipe(int level, int nSweeps, bool symmetric)
{
    LevelAddr& L = mesh->lev[level];
    Colouring& C = L.mc;
    const int key = nSweeps * 2 + (symmetric ? 1 : 0);
    if (C.pipe.count(key)) return;
    Colouring::Pipe& M = C.pipe[key];
    if (nSweeps < 1 || L.nCells == 0 || C.nColours == 0 || !C.tuned) return;
    if (L.nCells > k::kPipeMaxRanks * static_cast<int>(kPipeSmemCap / sizeof(float))) return;
    allowPipeSmem<float>();
    float* x = level == 0 ? w32.p : v32.corr[level - 1].p;
    float* b = level == 0 ? r32.p : v32.src[level - 1].p;
    // scratch vectors of the level (the times do not depend on the values)
    B2G_CUDA(cudaMemsetAsync(x, 0, sizeof(float) * static_cast<size_t>(nAlloc(level)), stream));
    B2G_CUDA(cudaMemsetAsync(b, 0, sizeof(float) * static_cast<size_t>(nAlloc(level)), stream));
    cudaEvent_t e0, e1;
    B2G_CUDA(cudaEventCreate(&e0));
    B2G_CUDA(cudaEventCreate(&e1));
    const long long l0 = launches;
    auto timeIt = [&](auto&& launch) {
        launch();  // warm
        B2G_CUDA(cudaEventRecord(e0, stream));
        for (int i = 0; i < 3; ++i) launch();
        B2G_CUDA(cudaEventRecord(e1, stream));
        B2G_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        B2G_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms / 3.f;
    };
    M.msColours = timeIt([&] { mcLaunch(level, C.fused, C.cluster, C.block, x, b, nSweeps, false, symmetric); });
    checkDeviceError();
    const LevelHost H = download(L, stream);
    const std::vector<int> rowPos = C.pos.download(stream);
    float best = M.msColours;
    for (int R : {1, 2, 4, 8, 16})
    {
        std::unique_ptr<PipeSchedule> P = colourSchedule(H, C, rowPos, nSweeps, symmetric, R, stream);
        if (!P) continue;
        if (R > 1 && !pipeClusterFits<float>(R, pipeSmemBytes(*P, sizeof(float)), stream, true)) continue;
        const float ms = timeIt([&] { pipeLaunch<float>(level, *P, x, b, true); });
        if (M.msPipe == 0.f || ms < M.msPipe) M.msPipe = ms;
        if (ms < best)
        {
            best = ms;
            M.sched = std::move(P);
            M.use = true;
        }
    }
    launches = l0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    B2G_CUDA(cudaStreamSynchronize(stream));
    checkDeviceError();
}

// Before a capture: the item blobs of every item-schedule choice, filled for the current
// coefficients.
template <class T>
void Matrix::refreshItems()
{
    for (int lv = 0; lv <= nLevels(); ++lv)
        for (auto& kv : mesh->lev[lv].pipe)
        {
            if (kv.first % 16 != static_cast<int>(sizeof(T))) continue;
            if (kv.second.mode == 2) itemBuffers<T>(lv, *kv.second.items);
        }
}

// nSweeps sweeps of `level` in one pipelined launch when the level's tuned choice says so; false
// when the sweeps run sweep by sweep (or the choice is not made yet and a capture is on).
template <class T>
bool Matrix::pipeSweeps(int level, T* psiL, const T* src, int nSweeps)
{
    LevelAddr& L = mesh->lev[level];
    auto it = L.pipe.find(pipeKey(nSweeps, sizeof(T)));
    if (it == L.pipe.end())
    {
        if (capturing || !g_pipeline) return false;
        ensurePipe<T>(level, nSweeps);
        it = L.pipe.find(pipeKey(nSweeps, sizeof(T)));
    }
    if (!g_pipeline) return false;
    const PipeChoice& C = it->second;
    if (C.mode == 1)
    {
        pipeLaunch<T>(level, *C.sched, psiL, src);
        return true;
    }
    if (C.mode == 2)
    {
        itemsLaunch<T>(level, *C.items, psiL, src);
        return true;
    }
    return false;
}

// A pipelined smoothing call on a given number of ranks, whatever the tuned choice (for tests):
// false when the level's cells do not fit that many CTAs or such a cluster cannot be resident.
template <class T>
bool Matrix::pipeForced(int level, T* psiL, const T* src, int nSweeps, int ranks)
{
    const LevelAddr& L = mesh->lev[level];
    if (nSweeps < 1 || L.nCells == 0) return false;
    if (ranks < 0)
    {
        // the item schedule, built for this call; its buffers on this matrix are dropped after it
        std::unique_ptr<GsSchedule> G = buildGsItems(L, nSweeps, stream);
        if (!G) return false;
        data<T>().items.erase(std::make_pair(level, nSweeps));
        itemsLaunch<T>(level, *G, psiL, src);
        B2G_CUDA(cudaStreamSynchronize(stream));
        data<T>().items.erase(std::make_pair(level, nSweeps));
        checkDeviceError();
        return true;
    }
    allowPipeSmem<T>();
    const LevelHost H = download(L, stream);
    int nSteps = 0;
    const std::vector<int> Tsteps = combinedSteps(H, nSweeps, nSteps);
    const bool grid = ranks > k::kPipeMaxRanks;
    if (grid && ranks > L.nCells) return false;
    std::unique_ptr<PipeSchedule> P = assemble(H, Tsteps, nSweeps, nSteps, ranks, sizeof(T), stream, grid);
    if (!P) return false;
    if (grid && !pipeGridFits<T>(ranks, pipeSmemBytes(*P, sizeof(T)))) return false;
    if (!grid && ranks > 1 && !pipeClusterFits<T>(ranks, pipeSmemBytes(*P, sizeof(T)), stream)) return false;
    pipeLaunch<T>(level, *P, psiL, src);
    B2G_CUDA(cudaStreamSynchronize(stream));  // P is released on return
    checkDeviceError();
    return true;
}

const PipeSchedule* pipeOneCta(LevelAddr& L, int S, size_t valueBytes, cudaStream_t s)
{
    const int key = pipeKey(S, valueBytes);
    auto it = L.pipeOne.find(key);
    if (it != L.pipeOne.end()) return it->second.get();
    std::unique_ptr<PipeSchedule>& P = L.pipeOne[key];
    if (S < 1 || L.nCells == 0 || static_cast<size_t>(L.nCells) * valueBytes > kPipeSmemCap) return nullptr;
    const LevelHost H = download(L, s);
    int nSteps = 0;
    const std::vector<int> Tsteps = combinedSteps(H, S, nSteps);
    P = assemble(H, Tsteps, S, nSteps, 1, valueBytes, s);
    return P.get();
}

// The batched one-CTA launch's shared-memory ceiling, once per device and value type.
template <class T>
static void allowPipeBatchSmem()
{
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    B2G_CUDA(cudaGetDevice(&dev));
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load() & bit) return;
    B2G_CUDA(cudaFuncSetAttribute(k::gsPipeBatch<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(kPipeSmemCap)));
    done.fetch_or(bit);
}
template <class T>
void launchPipeBatch(const void* table, const int* caseOf, int n, size_t smem, const int* active, cudaStream_t s)
{
    allowPipeBatchSmem<T>();
    k::gsPipeBatch<T><<<n, k::kPipeBlock, smem, s>>>(static_cast<const k::PipeArgs<T>*>(table), caseOf, active);
    B2G_LAUNCH_CHECK();
}
template void launchPipeBatch<double>(const void*, const int*, int, size_t, const int*, cudaStream_t);
template void launchPipeBatch<float>(const void*, const int*, int, size_t, const int*, cudaStream_t);

template void Matrix::ensurePipe<double>(int, int);
template bool Matrix::pipeForced<double>(int, double*, const double*, int, int);
template void Matrix::ensurePipe<float>(int, int);
template bool Matrix::pipeSweeps<double>(int, double*, const double*, int);
template bool Matrix::pipeSweeps<float>(int, float*, const float*, int);
template void Matrix::pipeLaunch<double>(int, const PipeSchedule&, double*, const double*, bool);
template void Matrix::pipeLaunch<float>(int, const PipeSchedule&, float*, const float*, bool);
template void Matrix::refreshItems<double>();
template k::PipeArgs<double> Matrix::pipeArgs<double>(int, const PipeSchedule&, double*, const double*);
template k::PipeArgs<float> Matrix::pipeArgs<float>(int, const PipeSchedule&, float*, const float*);
template void Matrix::refreshItems<float>();
template void Matrix::itemsLaunch<double>(int, const GsSchedule&, double*, const double*);

}  // namespace b2g
