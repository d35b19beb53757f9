// pair.cu -- the coupled (cyclic) pair on every level of a hierarchy and its coefficients for one
// matrix: what GAMGSolver carries through its interfaces on the standalone solve with a coupled patch.
//
// The finest level's pair is the coupled patches' faces, each once from its own side: faceCells and
// the neighbour cells face for face (gamgLevel0Interface, GAMG:440-470). A coarse level's pair is the
// finer one's keyed on the coarse cell pair (restrict[own], restrict[nbr]) in face order: the first
// face of a pair appends a coarse face, later ones merge into it, and the coarse coefficient is the sum
// of the merged fine ones from zero in ascending fine-face order (agglomerateMatrix, GAMG:497-524).
// The topology is built once per mesh on the host (pair faces are boundary faces: few against the
// cells); the coefficients are restricted on the device for every matrix.
//
// Reference: GAMG = src/matrices/lduMatrix/solvers/GAMG/gamg_solver_cpp.cu
#include "solver.cuh"

#include <algorithm>
#include <cstdint>
#include <string>
#include <unordered_map>

namespace b2g {

namespace {

constexpr int TPB = 256;

int gridFor(long long n) { return std::max(1, std::min(ceilDiv(n, TPB), 4096)); }

__global__ void kGatherInt(int n, const int* __restrict__ idx, const int* __restrict__ src, int* __restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = src[idx[i]];
}

// a coarse pair face's coefficient: its fine faces' summed from zero, ascending (GAMG:520-522)
__global__ void kPairRestrict(int nCoarse, const int* __restrict__ start, const int* __restrict__ list,
                              const double* __restrict__ fine, double* __restrict__ coarse)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nCoarse; c += gridDim.x * blockDim.x)
    {
        double acc = 0.0;
        for (int e = start[c]; e < start[c + 1]; ++e) acc = __dadd_rn(acc, fine[list[e]]);
        coarse[c] = acc;
    }
}

// the row layout's pair coefficient per entry
__global__ void kPairEntries(int n, const int* __restrict__ face, const double* __restrict__ coef,
                             double* __restrict__ val)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) val[k] = coef[face[k]];
}

// src[idx[i]] for host indices, through the device (the maps live there)
std::vector<int> gatherToHost(const std::vector<int>& idx, const int* dSrc, cudaStream_t s)
{
    const int n = static_cast<int>(idx.size());
    DBuf<int> di, dout;
    di.upload(idx.data(), idx.size(), s);
    dout.alloc(std::max(n, 1), s);
    if (n) kGatherInt<<<gridFor(n), TPB, 0, s>>>(n, di.p, dSrc, dout.p);
    B2G_LAUNCH_CHECK();
    std::vector<int> h = dout.download(s);
    h.resize(idx.size());
    return h;
}

}  // namespace

void buildPair(Mesh& M, int nFaces, const int* own, const int* nbr)
{
    if (M.hasPair) fail(B2G_ERR_STATE, "b2g: the mesh already carries a coupled pair.");
    if (nFaces <= 0) fail(B2G_ERR_ARGUMENT, "b2g: a coupled pair needs at least one face.");
    cudaStream_t s = M.stream;
    const int n0 = M.lev[0].nCells;
    std::vector<int> o(own, own + nFaces), nb(nbr, nbr + nFaces);
    for (int f = 0; f < nFaces; ++f)
        if (o[f] < 0 || o[f] >= n0 || nb[f] < 0 || nb[f] >= n0)
            fail(B2G_ERR_ARGUMENT, "b2g: coupled pair face " + std::to_string(f) + " names a cell outside the mesh.");
    for (int l = 0; l <= M.nLevels(); ++l)
    {
        LevelAddr& L = M.lev[l];
        PairLevel& P = L.pair;
        const int nF = static_cast<int>(o.size());
        P.nFaces = nF;
        P.own = o;
        P.nbr = nb;
        // the rows' pair entries: by the owner's position, the faces it owns in face order
        const std::vector<int> pOwn = gatherToHost(o, L.gs.posOf.p, s);
        const std::vector<int> pNbr = gatherToHost(nb, L.gs.posOf.p, s);
        std::vector<int> start(static_cast<size_t>(L.nCells) + 1, 0);
        for (int f = 0; f < nF; ++f) ++start[static_cast<size_t>(pOwn[f]) + 1];
        for (int c = 0; c < L.nCells; ++c) start[c + 1] += start[c];
        std::vector<int> fill(start.begin(), start.end() - 1), col(nF), face(nF);
        for (int f = 0; f < nF; ++f)
        {
            const int k = fill[pOwn[f]]++;
            col[k] = pNbr[f];
            face[k] = f;
        }
        P.start.upload(start.data(), start.size(), s);
        P.col.upload(col.data(), col.size(), s);
        P.face.upload(face.data(), face.size(), s);
        if (l == M.nLevels()) break;
        // the next level's pair, keyed on the coarse cell pair in face order (GAMG:505-523)
        const Step& S = M.step[l];
        const std::vector<int> co = gatherToHost(o, S.restrictAddr.p, s);
        const std::vector<int> cn = gatherToHost(nb, S.restrictAddr.p, s);
        std::unordered_map<uint64_t, int> seen;
        seen.reserve(static_cast<size_t>(nF) * 2);
        std::vector<int> nextOwn, nextNbr, toCoarse(nF);
        for (int f = 0; f < nF; ++f)
        {
            const uint64_t key = (static_cast<uint64_t>(static_cast<uint32_t>(co[f])) << 32) |
                                 static_cast<uint32_t>(cn[f]);
            auto it = seen.find(key);
            if (it == seen.end())
            {
                it = seen.emplace(key, static_cast<int>(nextOwn.size())).first;
                nextOwn.push_back(co[f]);
                nextNbr.push_back(cn[f]);
            }
            toCoarse[f] = it->second;
        }
        // coarse face -> its fine faces, ascending
        const int nC = static_cast<int>(nextOwn.size());
        std::vector<int> fStart(static_cast<size_t>(nC) + 1, 0), fList(nF);
        for (int f = 0; f < nF; ++f) ++fStart[static_cast<size_t>(toCoarse[f]) + 1];
        for (int c = 0; c < nC; ++c) fStart[c + 1] += fStart[c];
        std::vector<int> pos(fStart.begin(), fStart.end() - 1);
        for (int f = 0; f < nF; ++f) fList[pos[toCoarse[f]]++] = f;
        PairLevel& Q = M.lev[l + 1].pair;
        Q.fStart.upload(fStart.data(), fStart.size(), s);
        Q.fList.upload(fList.data(), fList.size(), s);
        o.swap(nextOwn);
        nb.swap(nextNbr);
    }
    B2G_CUDA(cudaStreamSynchronize(s));
    M.hasPair = true;
}

// The pair's coefficients on every level for this matrix: the finest level's as handed in (per pair
// face, in the order b2g_mesh_set_pair took the faces), each coarse level's restricted from the finer
// one, and every level's per row entry.
void Matrix::setPairCoeffs(const double* coeff, int memspace)
{
    if (!mesh->hasPair) fail(B2G_ERR_STATE, "b2g: the mesh carries no coupled pair (b2g_mesh_set_pair).");
    const int nL = nLevels();
    LevelCoef<double>& C0 = v64.coef[0];
    const int nF0 = mesh->lev[0].pair.nFaces;
    C0.pairCoef.alloc(static_cast<size_t>(std::max(nF0, 1)), stream);
    B2G_CUDA(cudaMemcpyAsync(C0.pairCoef.p, coeff, sizeof(double) * nF0,
                             memspace == B2G_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, stream));
    for (int l = 1; l <= nL; ++l)
    {
        const PairLevel& P = mesh->lev[l].pair;
        LevelCoef<double>& C = v64.coef[l];
        C.pairCoef.alloc(static_cast<size_t>(std::max(P.nFaces, 1)), stream);
        kPairRestrict<<<gridFor(P.nFaces), TPB, 0, stream>>>(P.nFaces, P.fStart.p, P.fList.p,
                                                              v64.coef[l - 1].pairCoef.p, C.pairCoef.p);
        B2G_LAUNCH_CHECK();
    }
    for (int l = 0; l <= nL; ++l)
    {
        const PairLevel& P = mesh->lev[l].pair;
        LevelCoef<double>& C = v64.coef[l];
        C.pairVal.alloc(static_cast<size_t>(std::max(P.nFaces, 1)), stream);
        kPairEntries<<<gridFor(P.nFaces), TPB, 0, stream>>>(P.nFaces, P.face.p, C.pairCoef.p, C.pairVal.p);
        B2G_LAUNCH_CHECK();
    }
    coupled = true;
}

}  // namespace b2g
