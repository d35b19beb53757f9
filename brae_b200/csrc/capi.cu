// capi.cu -- the extern "C" boundary (include/brae_gamg.h): handles, status codes, the last-error
// string, host/device argument staging, and the fvSolution entry reader with the reference's
// refusals (readGamgControls, src/matrices/lduMatrix/solvers/GAMG/gamg_solver_cpp.cu:801-928, and
// the PCG keys of src/applications/solvers/interFoam/inter_case_cpp.cu:1519-1572).
#include "capi_internal.cuh"

#include <cctype>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>

namespace b2g {
namespace capi {

thread_local std::string lastError;

void need(bool ok, const char* msg)
{
    if (!ok) b2g::fail(B2G_ERR_ARGUMENT, msg);
}

}  // namespace capi
}  // namespace b2g

namespace {

using b2g::capi::guarded;
using b2g::capi::need;

cudaStream_t streamOf(void* s) { return s ? static_cast<cudaStream_t>(s) : cudaStreamPerThread; }

// ---------------------------------------------------------------------------------------------
// the hierarchy cache: a content signature of the agglomeration's inputs and the file that keeps
// each step's restriction map
// ---------------------------------------------------------------------------------------------

__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    // the SplitMix64 finaliser
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// XOR of a hash of every (array, index, word): independent of the order the threads run in
__global__ void kSignature(long long nWords, const unsigned* __restrict__ words, unsigned long long salt,
                           unsigned long long* __restrict__ out)
{
    unsigned long long acc = 0ull;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nWords; i += (long long)gridDim.x * blockDim.x)
        acc ^= mix64(salt ^ mix64(static_cast<unsigned long long>(i) * 0x9e3779b97f4a7c15ull + words[i]));
    for (int o = 16; o > 0; o >>= 1) acc ^= __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicXor(out, acc);
}

unsigned long long meshSignature(int nCells, int nFaces, const int* lower, const int* upper, const double* Sf,
                                 const double* magSf, int nCoarsest, int forward, cudaStream_t s)
{
    b2g::DBuf<unsigned long long> acc;
    acc.alloc(1, s);
    acc.zero(s);
    const struct
    {
        const void* p;
        long long words;
        unsigned long long salt;
    } arrays[] = {{lower, nFaces, 0x6c6f776572ull}, {upper, nFaces, 0x7570706572ull},
                  {Sf, 6LL * nFaces, 0x5366ull}, {magSf, 2LL * nFaces, 0x6d61675366ull}};
    for (const auto& a : arrays)
        if (a.words)
            kSignature<<<std::min<long long>(b2g::ceilDiv(a.words, 256), 4096), 256, 0, s>>>(
                a.words, static_cast<const unsigned*>(a.p), a.salt, acc.p);
    B2G_LAUNCH_CHECK();
    unsigned long long h = 0;
    B2G_CUDA(cudaMemcpyAsync(&h, acc.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    B2G_CUDA(cudaStreamSynchronize(s));
    // the sizes and controls that also decide the agglomeration
    const unsigned long long scal[4] = {static_cast<unsigned long long>(nCells), static_cast<unsigned long long>(nFaces),
                                        static_cast<unsigned long long>(nCoarsest),
                                        static_cast<unsigned long long>(forward ? 1 : 0)};
    for (unsigned long long v : scal) h = (h ^ v) * 0x100000001b3ull + 0x9e3779b97f4a7c15ull;
    return h;
}

struct CachedAgglomeration
{
    int forwardOut = 1;
    std::vector<std::vector<int>> maps;
    std::vector<int> nCoarse;
};

constexpr char kCacheMagic[8] = {'B', '2', 'G', 'A', 'G', 'G', '0', '1'};

// The file: magic, signature, the direction flag after agglomerating, the step count, then per step
// nFine, nCoarse and the restriction map. False when it is missing, unreadable or for other inputs.
bool readCache(const char* path, unsigned long long sig, CachedAgglomeration& ca)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    bool ok = false;
    char magic[8];
    unsigned long long fsig = 0;
    int hdr[2] = {0, 0};
    if (std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kCacheMagic, 8) == 0 &&
        std::fread(&fsig, sizeof(fsig), 1, f) == 1 && fsig == sig && std::fread(hdr, sizeof(int), 2, f) == 2 &&
        hdr[1] >= 0 && hdr[1] < 64)
    {
        ca.forwardOut = hdr[0];
        ok = true;
        for (int i = 0; i < hdr[1] && ok; ++i)
        {
            int sz[2];
            if (std::fread(sz, sizeof(int), 2, f) != 2 || sz[0] < 0 || sz[1] < 1) { ok = false; break; }
            std::vector<int> m(static_cast<size_t>(sz[0]));
            if (sz[0] && std::fread(m.data(), sizeof(int), m.size(), f) != m.size()) { ok = false; break; }
            for (int v : m)
                if (v < 0 || v >= sz[1]) { ok = false; break; }
            ca.maps.push_back(std::move(m));
            ca.nCoarse.push_back(sz[1]);
        }
    }
    std::fclose(f);
    if (!ok) ca = CachedAgglomeration{};
    return ok;
}

void writeCache(const char* path, unsigned long long sig, const CachedAgglomeration& ca)
{
    FILE* f = std::fopen(path, "wb");
    if (!f) b2g::fail(B2G_ERR_STATE, std::string("b2g_mesh_create_cached: cannot write ") + path);
    bool ok = std::fwrite(kCacheMagic, 1, 8, f) == 8 && std::fwrite(&sig, sizeof(sig), 1, f) == 1;
    const int hdr[2] = {ca.forwardOut, static_cast<int>(ca.maps.size())};
    ok = ok && std::fwrite(hdr, sizeof(int), 2, f) == 2;
    for (size_t i = 0; i < ca.maps.size() && ok; ++i)
    {
        const int sz[2] = {static_cast<int>(ca.maps[i].size()), ca.nCoarse[i]};
        ok = std::fwrite(sz, sizeof(int), 2, f) == 2 &&
             std::fwrite(ca.maps[i].data(), sizeof(int), ca.maps[i].size(), f) == ca.maps[i].size();
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) b2g::fail(B2G_ERR_STATE, std::string("b2g_mesh_create_cached: cannot write ") + path);
}

__global__ void kCheckCells(int n, int nCells, const int* __restrict__ cells, int* __restrict__ err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && (cells[i] < 0 || cells[i] >= nCells)) atomicOr(err, 1);
}

__global__ void kIotaInt(int n, int* __restrict__ v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

// foldBoundary (gamg_solver_cpp.cu:769-797) per cell: its boundary faces in (patch, face) order,
// every patch's internal coefficient onto the diagonal, the uncoupled patches' boundary coefficient
// onto the source, one after another as the reference's loop adds them
__global__ void kFold(int nCells, const int* __restrict__ start, const int* __restrict__ order,
                      const double* __restrict__ ic, const double* __restrict__ bc,
                      const unsigned char* __restrict__ coupled, double* __restrict__ diag,
                      double* __restrict__ source)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nCells) return;
    const int e0 = start[c], e1 = start[c + 1];
    if (e0 == e1) return;
    double d = diag[c], s = source[c];
    for (int e = e0; e < e1; ++e)
    {
        const int i = order[e];
        d = __dadd_rn(d, ic[i]);
        if (!coupled[i]) s = __dadd_rn(s, bc[i]);
    }
    diag[c] = d;
    source[c] = s;
}

template <class T>
void stage(b2g::DBuf<T>& d, const T* src, size_t n, int memspace, cudaStream_t s)
{
    d.alloc(n, s);
    if (!n) return;
    B2G_CUDA(cudaMemcpyAsync(d.p, src, n * sizeof(T),
                             memspace == B2G_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
}

// ---------------------------------------------------------------------------------------------
// a minimal OpenFOAM dictionary: `key value;` and `key { ... }`, with // and /* */ comments
// ---------------------------------------------------------------------------------------------

struct Dict
{
    std::map<std::string, std::string> words;
    std::map<std::string, std::unique_ptr<Dict>> subs;
    bool found(const std::string& k) const { return words.count(k) || subs.count(k); }
    const Dict* sub(const std::string& k) const
    {
        auto it = subs.find(k);
        return it == subs.end() ? nullptr : it->second.get();
    }
    std::string wordOr(const std::string& k, const std::string& d) const
    {
        auto it = words.find(k);
        return it == words.end() ? d : it->second;
    }
};

std::vector<std::string> tokenize(const std::string& t)
{
    std::vector<std::string> out;
    size_t i = 0;
    while (i < t.size())
    {
        const char c = t[i];
        if (std::isspace(static_cast<unsigned char>(c))) { ++i; continue; }
        if (c == '/' && i + 1 < t.size() && t[i + 1] == '/')
        {
            while (i < t.size() && t[i] != '\n') ++i;
            continue;
        }
        if (c == '/' && i + 1 < t.size() && t[i + 1] == '*')
        {
            const size_t e = t.find("*/", i + 2);
            i = e == std::string::npos ? t.size() : e + 2;
            continue;
        }
        if (c == '{' || c == '}' || c == ';')
        {
            out.emplace_back(1, c);
            ++i;
            continue;
        }
        if (c == '"')
        {
            const size_t e = t.find('"', i + 1);
            out.push_back(t.substr(i + 1, (e == std::string::npos ? t.size() : e) - i - 1));
            i = e == std::string::npos ? t.size() : e + 1;
            continue;
        }
        size_t j = i;
        while (j < t.size() && !std::isspace(static_cast<unsigned char>(t[j])) && t[j] != '{' && t[j] != '}' &&
               t[j] != ';')
            ++j;
        out.push_back(t.substr(i, j - i));
        i = j;
    }
    return out;
}

void parseInto(Dict& d, const std::vector<std::string>& tok, size_t& i, bool nested)
{
    while (i < tok.size())
    {
        if (tok[i] == "}")
        {
            if (!nested) b2g::fail(B2G_ERR_ARGUMENT, "b2g: unbalanced '}' in the solver entry.");
            ++i;
            return;
        }
        if (tok[i] == ";") { ++i; continue; }
        const std::string key = tok[i++];
        if (i < tok.size() && tok[i] == "{")
        {
            ++i;
            auto sub = std::make_unique<Dict>();
            parseInto(*sub, tok, i, true);
            d.subs[key] = std::move(sub);
            continue;
        }
        std::string val;
        while (i < tok.size() && tok[i] != ";" && tok[i] != "}")
        {
            if (!val.empty()) val += ' ';
            val += tok[i++];
        }
        if (i < tok.size() && tok[i] == ";") ++i;
        d.words[key] = val;
    }
    if (nested) b2g::fail(B2G_ERR_ARGUMENT, "b2g: unbalanced '{' in the solver entry.");
}

double scalarOr(const Dict& d, const std::string& k, double def, const std::string& who)
{
    if (!d.words.count(k)) return def;
    const std::string v = d.wordOr(k, "");
    char* end = nullptr;
    const double x = std::strtod(v.c_str(), &end);
    if (end == v.c_str() || *end != '\0') b2g::fail(B2G_ERR_ARGUMENT, who + "has `" + k + " " + v + "`, not a number.");
    return x;
}

int intOr(const Dict& d, const std::string& k, int def, const std::string& who)
{
    return static_cast<int>(scalarOr(d, k, def, who));
}

bool switchOr(const Dict& d, const std::string& k, bool def, const std::string& who)
{
    if (!d.found(k)) return def;
    const std::string w = d.wordOr(k, "");
    if (w == "yes" || w == "true" || w == "on" || w == "y" || w == "t" || w == "1") return true;
    if (w == "no" || w == "false" || w == "off" || w == "n" || w == "f" || w == "0") return false;
    b2g::fail(B2G_ERR_REFUSED, who + "has `" + k + " " + w + "`, which is not a Switch.");
}

// readGamgControls (gamg_solver_cpp.cu:801-928) on a GAMG dictionary
void readGamg(const Dict& d, b2g_controls& c, const std::string& who)
{
    const std::string sm = d.wordOr("smoother", "");
    if (sm.empty())
        b2g::fail(B2G_ERR_REFUSED, who + "names no `smoother`. lduMatrix::smoother::New reads it with a mandatory "
                                         "lookup and OpenFOAM stops without it.");
    if (sm == "GaussSeidel") c.smoother = B2G_SMOOTHER_GAUSS_SEIDEL;
    else if (sm == "symGaussSeidel") c.smoother = B2G_SMOOTHER_SYM_GAUSS_SEIDEL;
    else if (sm == "DIC") c.smoother = B2G_SMOOTHER_DIC;
    else if (sm == "DICGaussSeidel") c.smoother = B2G_SMOOTHER_DIC_GAUSS_SEIDEL;
    else if (sm == "DILU" || sm == "DILUGaussSeidel")
        b2g::fail(B2G_ERR_REFUSED,
                  who + "asks for `smoother " + sm + "`, which OpenFOAM registers for an ASYMMETRIC matrix only. "
                  "This matrix is symmetric, so OpenFOAM's own lookup stops: `Unknown symmetric matrix smoother "
                  "type " + sm + "`. The symmetric smoothers are DIC, DICGaussSeidel, FDIC, GaussSeidel, "
                  "symGaussSeidel and nonBlockingGaussSeidel.");
    else
        b2g::fail(B2G_ERR_REFUSED,
                  who + "asks for `smoother " + sm + "`, which is not ported: DIC, DICGaussSeidel, GaussSeidel and "
                  "symGaussSeidel are." +
                      ((sm == "FDIC" || sm == "nonBlockingGaussSeidel")
                           ? std::string(" OpenFOAM does accept it on a symmetric matrix.")
                           : std::string(" OpenFOAM has no smoother of that name either.")));
    c.nPreSweeps = intOr(d, "nPreSweeps", c.nPreSweeps, who);
    c.preSweepsLevelMultiplier = intOr(d, "preSweepsLevelMultiplier", c.preSweepsLevelMultiplier, who);
    c.maxPreSweeps = intOr(d, "maxPreSweeps", c.maxPreSweeps, who);
    c.nPostSweeps = intOr(d, "nPostSweeps", c.nPostSweeps, who);
    c.postSweepsLevelMultiplier = intOr(d, "postSweepsLevelMultiplier", c.postSweepsLevelMultiplier, who);
    c.maxPostSweeps = intOr(d, "maxPostSweeps", c.maxPostSweeps, who);
    c.nFinestSweeps = intOr(d, "nFinestSweeps", c.nFinestSweeps, who);
    c.scaleCorrection = switchOr(d, "scaleCorrection", true, who) ? 1 : 0;
    c.nCellsInCoarsestLevel = intOr(d, "nCellsInCoarsestLevel", 10, who);
    const std::string agg = d.wordOr("agglomerator", "faceAreaPair");
    if (agg != "faceAreaPair")
        b2g::fail(B2G_ERR_REFUSED, who + "asks for `agglomerator " + agg + "`. Only faceAreaPair is built; another "
                                         "agglomerator is another hierarchy.");
    if (intOr(d, "mergeLevels", 1, who) != 1)
        b2g::fail(B2G_ERR_REFUSED, who + "asks for `mergeLevels " + d.wordOr("mergeLevels", "") +
                                         "`. pairGAMGAgglomeration then folds pairs of levels into one "
                                         "(combineLevels), which is not built.");
    if (intOr(d, "updateInterval", 1, who) != 1)
        b2g::fail(B2G_ERR_REFUSED, who + "sets `updateInterval`. faceAreaPairGAMGAgglomeration then weighs faces by "
                                         "magSf off the update steps; only the default's branch is built.");
    if (!switchOr(d, "cacheAgglomeration", true, who))
        b2g::fail(B2G_ERR_REFUSED, who + "sets `cacheAgglomeration no`. The hierarchy is then rebuilt at every solve "
                                         "from wherever the static pairing direction was left; it is built once here.");
    if (switchOr(d, "interpolateCorrection", false, who))
        b2g::fail(B2G_ERR_REFUSED, who + "sets `interpolateCorrection yes` (GAMGSolverInterpolate.C), which is not built.");
    if (switchOr(d, "directSolveCoarsest", false, who))
        b2g::fail(B2G_ERR_REFUSED, who + "sets `directSolveCoarsest yes`. The coarsest level is then LU-factored rather "
                                         "than solved by PCG to the entry's tolerance (GAMGSolver.C:303), which is "
                                         "not built.");
    if (d.sub("coarsestLevelCorr"))
        b2g::fail(B2G_ERR_REFUSED, who + "carries a `coarsestLevelCorr` sub-dictionary. GAMGSolver then builds the "
                                         "coarsest level's solver from it instead of PCG with DIC at the entry's own "
                                         "tolerance.");
    if (d.found("processorAgglomerator"))
        b2g::fail(B2G_ERR_REFUSED, who + "names a `processorAgglomerator`. This is a serial solver.");
}

}  // namespace

namespace b2g {
namespace capi {

std::unique_ptr<b2g_mesh> createMesh(int nCells, int nFaces, const int32_t* lower, const int32_t* upper,
                                     const double* Sf, const double* magSf, int nCellsInCoarsestLevel,
                                     int* forwardInOut, int memspace, cudaStream_t stream, const char* cachePath,
                                     int* fromCache)
{
    need(nCells > 0 && nFaces >= 0, "b2g_mesh_create: nCells must be positive and nFaces non-negative");
    need(nFaces == 0 || (lower && upper && Sf && magSf), "b2g_mesh_create: null array");
    need(forwardInOut != nullptr, "b2g_mesh_create: null direction flag");
    need(memspace == B2G_MEM_HOST || memspace == B2G_MEM_DEVICE, "b2g_mesh_create: bad memspace");
    std::unique_ptr<b2g_mesh> h(new b2g_mesh);
    b2g::Mesh& M = h->m;
    M.stream = stream;
    cudaGetDevice(&M.device);
    cudaEvent_t e0, e1;
    B2G_CUDA(cudaEventCreate(&e0));
    B2G_CUDA(cudaEventCreate(&e1));
    B2G_CUDA(cudaEventRecord(e0, M.stream));
    M.lev.emplace_back();
    b2g::LevelAddr& L0 = M.lev[0];
    L0.nCells = nCells;
    L0.nFaces = nFaces;
    stage(L0.lower, lower, nFaces, memspace, M.stream);
    stage(L0.upper, upper, nFaces, memspace, M.stream);
    b2g::DBuf<double> dSf, dMag;
    stage(dSf, Sf, 3 * (size_t)nFaces, memspace, M.stream);
    stage(dMag, magSf, nFaces, memspace, M.stream);
    if (fromCache) *fromCache = 0;
    if (!cachePath)
    {
        b2g::buildHierarchy(M, dSf.p, dMag.p, nCellsInCoarsestLevel, forwardInOut);
    }
    else
    {
        const unsigned long long sig = meshSignature(nCells, nFaces, L0.lower.p, L0.upper.p, dSf.p, dMag.p,
                                                     nCellsInCoarsestLevel, *forwardInOut, M.stream);
        CachedAgglomeration ca;
        if (readCache(cachePath, sig, ca))
        {
            b2g::buildHierarchyFromMaps(M, dSf.p, dMag.p, ca.maps, ca.nCoarse);
            *forwardInOut = ca.forwardOut;
            if (fromCache) *fromCache = 1;
        }
        else
        {
            const int fwdIn = *forwardInOut;
            b2g::buildHierarchy(M, dSf.p, dMag.p, nCellsInCoarsestLevel, forwardInOut);
            ca.forwardOut = *forwardInOut;
            for (const b2g::Step& st : M.step)
            {
                ca.maps.push_back(st.restrictAddr.download(M.stream));
                ca.nCoarse.push_back(st.nCoarse);
            }
            (void)fwdIn;
            writeCache(cachePath, sig, ca);
        }
    }
    B2G_CUDA(cudaEventRecord(e1, M.stream));
    B2G_CUDA(cudaEventSynchronize(e1));
    B2G_CUDA(cudaEventElapsedTime(&M.buildMs, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return h;
}

// The host source and psi copied into A.fc / A.fr on the matrix's side stream, after the copies already
// queued on its stream (the matrix's coefficients) have crossed; joinSideCopies makes the stream wait.
void stageSideCopies(b2g::Matrix& A, const double* source, const double* psi)
{
    if (!A.sideStream)
    {
        B2G_CUDA(cudaStreamCreateWithFlags(&A.sideStream, cudaStreamNonBlocking));
        B2G_CUDA(cudaEventCreateWithFlags(&A.sideEv[0], cudaEventDisableTiming));
        B2G_CUDA(cudaEventCreateWithFlags(&A.sideEv[1], cudaEventDisableTiming));
    }
    const size_t bytes = sizeof(double) * static_cast<size_t>(A.n(0));
    B2G_CUDA(cudaEventRecord(A.sideEv[0], A.stream));
    B2G_CUDA(cudaStreamWaitEvent(A.sideStream, A.sideEv[0], 0));
    B2G_CUDA(cudaMemcpyAsync(A.fc.p, source, bytes, cudaMemcpyHostToDevice, A.sideStream));
    B2G_CUDA(cudaMemcpyAsync(A.fr.p, psi, bytes, cudaMemcpyHostToDevice, A.sideStream));
    B2G_CUDA(cudaEventRecord(A.sideEv[1], A.sideStream));
}

void joinSideCopies(b2g::Matrix& A) { B2G_CUDA(cudaStreamWaitEvent(A.stream, A.sideEv[1], 0)); }

void solveOn(b2g::Matrix& A, const double* source, double* psi, const b2g_controls* c, int memspace,
             b2g_perf* out, b2g_solve_log* log, bool standalone, bool staged)
{
    need(c && source && psi && out, "b2g solve: null argument");
    need(memspace == B2G_MEM_HOST || memspace == B2G_MEM_DEVICE, "b2g solve: bad memspace");
    need(c->precision >= B2G_PRECISION_FP64 && c->precision <= B2G_PRECISION_FP32_PRECOND_MULTICOLOUR,
         "b2g solve: unknown precision form");
    if (A.coupled && !standalone)
        b2g::fail(B2G_ERR_REFUSED, "b2g: PCG with the GAMG preconditioner refuses coupled patches, as the reference's "
                                   "pcgGamgSolve does (gamg_solver_cpp.cu:1045); the standalone GAMG solve carries the "
                                   "pair (b2g_gamg_solve_coupled)");
    if (A.coupled && c->precision != B2G_PRECISION_FP64)
        b2g::fail(B2G_ERR_REFUSED, "b2g: a matrix with a coupled pair is solved in the FP64 form only");
    const int n0 = A.n(0);
    // the solve runs in the finest level's position order: host fields are staged in fc/fr (free
    // outside a solve) and permuted on the device; device fields are permuted in place of a copy
    if (memspace == B2G_MEM_HOST)
    {
        if (!staged)
        {
            B2G_CUDA(cudaMemcpyAsync(A.fc.p, source, sizeof(double) * n0, cudaMemcpyHostToDevice, A.stream));
            B2G_CUDA(cudaMemcpyAsync(A.fr.p, psi, sizeof(double) * n0, cudaMemcpyHostToDevice, A.stream));
        }
        A.toPos(0, static_cast<const double*>(A.fc.p), A.source.p);
        A.toPos(0, static_cast<const double*>(A.fr.p), A.psi.p);
    }
    else
    {
        A.toPos(0, source, A.source.p);
        A.toPos(0, static_cast<const double*>(psi), A.psi.p);
    }
    *out = standalone ? A.gamg(*c, log) : A.pcg(*c, log);
    if (memspace == B2G_MEM_HOST)
    {
        A.fromPos(0, static_cast<const double*>(A.psi.p), A.fc.p);
        B2G_CUDA(cudaMemcpyAsync(psi, A.fc.p, sizeof(double) * n0, cudaMemcpyDeviceToHost, A.stream));
    }
    else
    {
        A.fromPos(0, static_cast<const double*>(A.psi.p), psi);
    }
    B2G_CUDA(cudaStreamSynchronize(A.stream));
}

}  // namespace capi
}  // namespace b2g

extern "C" {

const char* b2g_last_error(void) { return b2g::capi::lastError.c_str(); }

const char* b2g_version(void) { return "brae_b200 0.1 (sm_100a)"; }

b2g_status b2g_set_profiling(int on)
{
    b2g::g_profiling = on != 0;
    return B2G_OK;
}

b2g_status b2g_set_sweep_pipeline(int on)
{
    b2g::g_pipeline = on != 0;
    return B2G_OK;
}

b2g_status b2g_set_part_cells(int cells)
{
    return guarded([&] {
        need(cells >= 1 && cells <= 65536, "b2g_set_part_cells: cells must be in [1, 65536]");
        b2g::g_partCells.store(cells);
    });
}

b2g_status b2g_controls_default(b2g_controls* out)
{
    return guarded([&] {
        need(out != nullptr, "b2g_controls_default: null output");
        b2g_controls c{};
        c.solver = B2G_SOLVER_PCG_GAMG;
        c.tolerance = 1e-6;
        c.relTol = 0.0;
        c.maxIter = 1000;
        c.minIter = 0;
        c.smoother = B2G_SMOOTHER_GAUSS_SEIDEL;
        c.precTolerance = 1e-6;
        c.precRelTol = 0.0;
        c.nPreSweeps = 0;
        c.preSweepsLevelMultiplier = 1;
        c.maxPreSweeps = 4;
        c.nPostSweeps = 2;
        c.postSweepsLevelMultiplier = 1;
        c.maxPostSweeps = 4;
        c.nFinestSweeps = 2;
        c.scaleCorrection = 1;
        c.nCellsInCoarsestLevel = 10;
        c.nVcycles = 2;
        c.precision = B2G_PRECISION_FP64;
        c.reduction = B2G_REDUCTION_TREE;
        c.coarsestDirect = 1;
        *out = c;
    });
}

b2g_status b2g_controls_read(const char* text, b2g_controls* out)
{
    return guarded([&] {
        need(text != nullptr && out != nullptr, "b2g_controls_read: null argument");
        b2g_controls c{};
        b2g_controls_default(&c);
        Dict d;
        const std::vector<std::string> tok = tokenize(text);
        size_t i = 0;
        parseInto(d, tok, i, false);
        const std::string who = "b2g: fvSolution's solver entry ";
        const std::string solver = d.wordOr("solver", "");
        // lduMatrix::solver::readControls: tolerance 1e-6, relTol 0, maxIter 1000 when absent
        c.tolerance = scalarOr(d, "tolerance", 1e-6, who);
        c.relTol = scalarOr(d, "relTol", 0.0, who);
        c.maxIter = static_cast<int>(scalarOr(d, "maxIter", 1000, who));
        c.minIter = intOr(d, "minIter", 0, who);
        if (solver == "GAMG")
        {
            c.solver = B2G_SOLVER_GAMG;
            readGamg(d, c, who);
            c.precTolerance = c.tolerance;
            c.precRelTol = c.relTol;
        }
        else if (solver == "PCG")
        {
            c.solver = B2G_SOLVER_PCG_GAMG;
            const Dict* pd = d.sub("preconditioner");
            if (!pd)
                b2g::fail(B2G_ERR_REFUSED,
                          who + "names `preconditioner " + d.wordOr("preconditioner", "") +
                              "`. This solver is PCG with a `preconditioner { preconditioner GAMG; ... }` "
                              "sub-dictionary, the form whose controls GAMG reads.");
            const std::string name = pd->wordOr("preconditioner", "");
            if (name != "GAMG")
                b2g::fail(B2G_ERR_REFUSED, who + "has `preconditioner { preconditioner " + name +
                                                 "; }`. Only the GAMG preconditioner is built here.");
            const std::string pwho = who + "(its GAMG preconditioner) ";
            readGamg(*pd, c, pwho);
            // lduMatrix::solver::readControls on the sub-dictionary: its own defaults
            c.precTolerance = scalarOr(*pd, "tolerance", 1e-6, pwho);
            c.precRelTol = scalarOr(*pd, "relTol", 0.0, pwho);
            c.nVcycles = intOr(*pd, "nVcycles", 2, pwho);
            if (c.nVcycles < 1) b2g::fail(B2G_ERR_REFUSED, "b2g GAMG preconditioner: nVcycles must be at least 1.");
        }
        else
        {
            b2g::fail(B2G_ERR_REFUSED, who + "names `solver " + solver + "`. This library solves `solver PCG;` with "
                                             "the GAMG preconditioner and `solver GAMG;`.");
        }
        *out = c;
    });
}

b2g_status b2g_mesh_create(int nCells, int nFaces, const int32_t* lower, const int32_t* upper, const double* Sf,
                           const double* magSf, int nCellsInCoarsestLevel, int* forwardInOut, int memspace,
                           void* stream, b2g_mesh** out)
{
    return guarded([&] {
        need(out != nullptr, "b2g_mesh_create: null output handle");
        *out = nullptr;
        *out = b2g::capi::createMesh(nCells, nFaces, lower, upper, Sf, magSf, nCellsInCoarsestLevel, forwardInOut,
                                     memspace, streamOf(stream))
                   .release();
    });
}

b2g_status b2g_mesh_create_cached(int nCells, int nFaces, const int32_t* lower, const int32_t* upper,
                                  const double* Sf, const double* magSf, int nCellsInCoarsestLevel, int* forwardInOut,
                                  int memspace, void* stream, const char* cachePath, b2g_mesh** out, int* fromCache)
{
    return guarded([&] {
        need(out != nullptr && cachePath != nullptr, "b2g_mesh_create_cached: null output handle or path");
        *out = nullptr;
        *out = b2g::capi::createMesh(nCells, nFaces, lower, upper, Sf, magSf, nCellsInCoarsestLevel, forwardInOut,
                                     memspace, streamOf(stream), cachePath, fromCache)
                   .release();
    });
}

b2g_status b2g_mesh_destroy(b2g_mesh* mesh)
{
    return guarded([&] {
        if (!mesh) return;
        cudaStream_t s = mesh->m.stream;
        delete mesh;
        B2G_CUDA(cudaStreamSynchronize(s));
    });
}

b2g_status b2g_mesh_levels(const b2g_mesh* mesh, int* nLevels)
{
    return guarded([&] {
        need(mesh && nLevels, "b2g_mesh_levels: null argument");
        *nLevels = mesh->m.nLevels();
    });
}

b2g_status b2g_mesh_level_size(const b2g_mesh* mesh, int level, int* nCells, int* nFaces)
{
    return guarded([&] {
        need(mesh && nCells && nFaces, "b2g_mesh_level_size: null argument");
        need(level >= 0 && level <= mesh->m.nLevels(), "b2g_mesh_level_size: level out of range");
        *nCells = mesh->m.lev[level].nCells;
        *nFaces = mesh->m.lev[level].nFaces;
    });
}

b2g_status b2g_mesh_get_step(const b2g_mesh* mesh, int step, int32_t* restrictAddr, int32_t* faceRestrict,
                             int8_t* flip, int32_t* coarseLower, int32_t* coarseUpper)
{
    return guarded([&] {
        need(mesh != nullptr, "b2g_mesh_get_step: null mesh");
        const b2g::Mesh& M = mesh->m;
        need(step >= 0 && step < M.nLevels(), "b2g_mesh_get_step: step out of range");
        const b2g::Step& S = M.step[step];
        const b2g::LevelAddr& C = M.lev[step + 1];
        cudaStream_t s = M.stream;
        if (restrictAddr)
            B2G_CUDA(cudaMemcpyAsync(restrictAddr, S.restrictAddr.p, sizeof(int) * S.nFine, cudaMemcpyDeviceToHost, s));
        if (faceRestrict && S.nFineFaces)
            B2G_CUDA(cudaMemcpyAsync(faceRestrict, S.faceRestrict.p, sizeof(int) * S.nFineFaces,
                                     cudaMemcpyDeviceToHost, s));
        if (flip && S.nFineFaces)
            B2G_CUDA(cudaMemcpyAsync(flip, S.flip.p, S.nFineFaces, cudaMemcpyDeviceToHost, s));
        if (coarseLower && C.nFaces)
            B2G_CUDA(cudaMemcpyAsync(coarseLower, C.lower.p, sizeof(int) * C.nFaces, cudaMemcpyDeviceToHost, s));
        if (coarseUpper && C.nFaces)
            B2G_CUDA(cudaMemcpyAsync(coarseUpper, C.upper.p, sizeof(int) * C.nFaces, cudaMemcpyDeviceToHost, s));
        B2G_CUDA(cudaStreamSynchronize(s));
    });
}

b2g_status b2g_mesh_build_ms(const b2g_mesh* mesh, float* ms)
{
    return guarded([&] {
        need(mesh && ms, "b2g_mesh_build_ms: null argument");
        *ms = mesh->m.buildMs;
    });
}

b2g_status b2g_matrix_create(b2g_mesh* mesh, const double* diag, const double* upper, int memspace, void* stream,
                             b2g_matrix** out)
{
    return guarded([&] {
        need(mesh && out && diag, "b2g_matrix_create: null argument");
        need(memspace == B2G_MEM_HOST || memspace == B2G_MEM_DEVICE, "b2g_matrix_create: bad memspace");
        need(mesh->m.lev[0].nFaces == 0 || upper, "b2g_matrix_create: null upper");
        std::unique_ptr<b2g_matrix> h(new b2g_matrix);
        h->mesh = mesh;
        (void)stream;
        h->mat.reset(new b2g::Matrix(&mesh->m, mesh->m.stream));
        h->mat->setFine(diag, upper, memspace);
        h->mat->buildCoarse();
        B2G_CUDA(cudaStreamSynchronize(mesh->m.stream));
        *out = h.release();
    });
}

b2g_status b2g_matrix_set_coeffs(b2g_matrix* m, const double* diag, const double* upper, int memspace)
{
    return guarded([&] {
        need(m && diag, "b2g_matrix_set_coeffs: null argument");
        need(memspace == B2G_MEM_HOST || memspace == B2G_MEM_DEVICE, "b2g_matrix_set_coeffs: bad memspace");
        need(m->mesh->m.lev[0].nFaces == 0 || upper, "b2g_matrix_set_coeffs: null upper");
        if (m->mat->coupled)
            b2g::fail(B2G_ERR_REFUSED, "b2g_matrix_set_coeffs: a matrix with a coupled pair takes new coefficients "
                                       "through b2g_matrix_create_coupled");
        m->mat->setFine(diag, upper, memspace);
        m->mat->buildCoarse();
        B2G_CUDA(cudaStreamSynchronize(m->mesh->m.stream));
    });
}

b2g_status b2g_matrix_destroy(b2g_matrix* m)
{
    return guarded([&] {
        if (!m) return;
        cudaStream_t s = m->mesh->m.stream;
        delete m;
        B2G_CUDA(cudaStreamSynchronize(s));
    });
}

b2g_status b2g_matrix_get_level(const b2g_matrix* m, int level, double* diag, double* upper)
{
    return guarded([&] {
        need(m != nullptr, "b2g_matrix_get_level: null matrix");
        const b2g::Matrix& A = *m->mat;
        need(level >= 0 && level <= A.nLevels(), "b2g_matrix_get_level: level out of range");
        const b2g::LevelAddr& L = A.mesh->lev[level];
        cudaStream_t s = A.stream;
        if (diag)
            B2G_CUDA(cudaMemcpyAsync(diag, A.v64.coef[level].diag.p, sizeof(double) * L.nCells, cudaMemcpyDeviceToHost, s));
        if (upper && L.nFaces)
            B2G_CUDA(cudaMemcpyAsync(upper, A.v64.coef[level].upper.p, sizeof(double) * L.nFaces,
                                     cudaMemcpyDeviceToHost, s));
        B2G_CUDA(cudaStreamSynchronize(s));
    });
}

b2g_status b2g_level_amul(b2g_matrix* m, int level, const double* x, double* y)
{
    return guarded([&] {
        need(m && x && y, "b2g_level_amul: null argument");
        need(level >= 0 && level <= m->mat->nLevels(), "b2g_level_amul: level out of range");
        b2g::Matrix& A = *m->mat;
        A.toPos(level, x, A.ioBuf(0));
        A.amul<double>(level, A.ioBuf(0), A.ioBuf(1));
        A.fromPos(level, static_cast<const double*>(A.ioBuf(1)), y);
        B2G_CUDA(cudaStreamSynchronize(A.stream));
    });
}

b2g_status b2g_level_smooth(b2g_matrix* m, int level, int smoother, double* psi, const double* source, int nSweeps)
{
    return guarded([&] {
        need(m && psi && source, "b2g_level_smooth: null argument");
        need(level >= 0 && level <= m->mat->nLevels(), "b2g_level_smooth: level out of range");
        b2g::Matrix& A = *m->mat;
        A.toPos(level, static_cast<const double*>(psi), A.ioBuf(0));
        A.toPos(level, source, A.ioBuf(1));
        A.smooth<double>(level, smoother, A.ioBuf(0), A.ioBuf(1), nSweeps);
        A.fromPos(level, static_cast<const double*>(A.ioBuf(0)), psi);
        A.checkDeviceError();
    });
}

b2g_status b2g_level_smooth_trace(b2g_matrix* m, int level, double* psi, const double* source,
                                  unsigned long long* trace, int traceCapacity, int* schedule)
{
    return guarded([&] {
        need(m && psi && source, "b2g_level_smooth_trace: null argument");
        need(level >= 0 && level <= m->mat->nLevels(), "b2g_level_smooth_trace: level out of range");
        const b2g::GsSchedule& G = m->mat->mesh->lev[level].gs;
        if (schedule)
        {
            schedule[0] = G.nParts;
            schedule[1] = G.nChunks;
            schedule[2] = G.maxCells;
            schedule[3] = G.maxEnt;
            schedule[4] = G.maxDepth;
        }
        need(trace == nullptr || traceCapacity >= 8LL * G.nChunks + 4LL * G.nParts + 2LL * G.nParts * (G.maxDepth + 2),
             "b2g_level_smooth_trace: trace too small");
        b2g::Matrix& A = *m->mat;
        A.toPos(level, static_cast<const double*>(psi), A.ioBuf(0));
        A.toPos(level, source, A.ioBuf(1));
        A.smooth<double>(level, B2G_SMOOTHER_GAUSS_SEIDEL, A.ioBuf(0), A.ioBuf(1), 1, trace);
        A.fromPos(level, static_cast<const double*>(A.ioBuf(0)), psi);
        A.checkDeviceError();
    });
}

b2g_status b2g_level_smooth_stall(b2g_matrix* m, int level, double* psi, const double* source, long long spinLimit,
                                  int* nParts)
{
    return guarded([&] {
        need(m && psi && source, "b2g_level_smooth_stall: null argument");
        need(level >= 0 && level <= m->mat->nLevels(), "b2g_level_smooth_stall: level out of range");
        need(spinLimit >= 1 && spinLimit <= b2g::k::kSpinLimit, "b2g_level_smooth_stall: spinLimit out of range");
        b2g::Matrix& A = *m->mat;
        const b2g::LevelAddr& L = A.mesh->lev[level];
        if (nParts) *nParts = L.gs.nParts;
        A.toPos(level, static_cast<const double*>(psi), A.ioBuf(0));
        A.toPos(level, source, A.ioBuf(1));
        A.spinLimit = spinLimit;
        A.publish = 0;
        try
        {
            A.gsLaunch<double>(L, A.v64.coef[level], A.ioBuf(0), A.ioBuf(1), nullptr, false);
        }
        catch (...)
        {
            A.spinLimit = b2g::k::kSpinLimit;
            A.publish = 1;
            throw;
        }
        A.spinLimit = b2g::k::kSpinLimit;
        A.publish = 1;
        A.fromPos(level, static_cast<const double*>(A.ioBuf(0)), psi);
        A.checkDeviceError();
    });
}

b2g_status b2g_level_grid_stall(b2g_matrix* m, int level, double* psi, const double* source, int nSweeps, int ranks,
                                long long spinLimit)
{
    return guarded([&] {
        need(m && psi && source, "b2g_level_grid_stall: null argument");
        need(level >= 0 && level <= m->mat->nLevels(), "b2g_level_grid_stall: level out of range");
        need(nSweeps >= 2, "b2g_level_grid_stall: nSweeps must be at least 2 (one step waits for another)");
        need(ranks > b2g::k::kPipeMaxRanks, "b2g_level_grid_stall: ranks must be above 16 (the grid form)");
        need(spinLimit >= 1 && spinLimit <= b2g::k::kSpinLimit, "b2g_level_grid_stall: spinLimit out of range");
        b2g::Matrix& A = *m->mat;
        need(!A.coupled, "b2g_level_grid_stall: not for a coupled matrix");
        A.toPos(level, static_cast<const double*>(psi), A.ioBuf(0));
        A.toPos(level, source, A.ioBuf(1));
        A.spinLimit = spinLimit;
        A.publish = 0;
        bool ran = false;
        try
        {
            ran = A.pipeForced<double>(level, A.ioBuf(0), A.ioBuf(1), nSweeps, ranks);
        }
        catch (...)
        {
            A.spinLimit = b2g::k::kSpinLimit;
            A.publish = 1;
            throw;
        }
        A.spinLimit = b2g::k::kSpinLimit;
        A.publish = 1;
        if (!ran) b2g::fail(B2G_ERR_ARGUMENT, "b2g_level_grid_stall: the level does not fit that many CTAs");
        A.fromPos(level, static_cast<const double*>(A.ioBuf(0)), psi);
        B2G_CUDA(cudaStreamSynchronize(A.stream));
    });
}

b2g_status b2g_level_smooth_pipelined(b2g_matrix* m, int level, double* psi, const double* source, int nSweeps,
                                      int ranks)
{
    return guarded([&] {
        need(m && psi && source, "b2g_level_smooth_pipelined: null argument");
        need(level >= 0 && level <= m->mat->nLevels(), "b2g_level_smooth_pipelined: level out of range");
        need(nSweeps >= 1, "b2g_level_smooth_pipelined: nSweeps must be positive");
        need(ranks == 1 || ranks == 2 || ranks == 4 || ranks == 8 || ranks == 16 || ranks == -1 || ranks > 16,
             "b2g_level_smooth_pipelined: ranks is 1, 2, 4, 8, 16, above 16 (the grid form) or -1 (the item "
             "schedule)");
        b2g::Matrix& A = *m->mat;
        need(!A.coupled, "b2g_level_smooth_pipelined: not for a coupled matrix");
        A.toPos(level, static_cast<const double*>(psi), A.ioBuf(0));
        A.toPos(level, source, A.ioBuf(1));
        if (!A.pipeForced<double>(level, A.ioBuf(0), A.ioBuf(1), nSweeps, ranks))
            b2g::fail(B2G_ERR_ARGUMENT, ranks < 0 ? "b2g_level_smooth_pipelined: the level has no item schedule "
                                                    "(one part, or one sweep)"
                                                  : "b2g_level_smooth_pipelined: the level does not fit that many CTAs");
        A.fromPos(level, static_cast<const double*>(A.ioBuf(0)), psi);
        B2G_CUDA(cudaStreamSynchronize(A.stream));
    });
}

b2g_status b2g_coarsest_dense_solve(b2g_matrix* m, double* psi, const double* source)
{
    return guarded([&] {
        need(m && psi && source, "b2g_coarsest_dense_solve: null argument");
        b2g::Matrix& A = *m->mat;
        const int lv = A.nLevels();
        need(lv > 0, "b2g_coarsest_dense_solve: the mesh has no coarse levels");
        A.ensureDense();
        if (!A.denseUse)
            b2g::fail(B2G_ERR_ARGUMENT, "b2g_coarsest_dense_solve: the coarsest level has no dense factor (more than "
                                        "96 cells, or not positive definite)");
        const int n = A.n(lv);
        A.toPos(lv, source, A.ioBuf(1));
        b2g::k::coarseDenseSolve<double><<<1, 32, sizeof(double) * n * n, A.stream>>>(n, A.denseL.p, A.ioBuf(1),
                                                                                       A.ioBuf(0));
        B2G_LAUNCH_CHECK();
        A.fromPos(lv, static_cast<const double*>(A.ioBuf(0)), psi);
        B2G_CUDA(cudaStreamSynchronize(A.stream));
    });
}

b2g_status b2g_level_pipe_shape(const b2g_mesh* mesh, int level, int nSweeps, int valueBytes, int* ranks,
                                int* nSteps, float* msPipe, float* msSweeps, float* msShared, float* msItems,
                                float* msGrid, int* gridForm)
{
    return guarded([&] {
        need(mesh != nullptr, "b2g_level_pipe_shape: null mesh");
        need(level >= 0 && level <= mesh->m.nLevels(), "b2g_level_pipe_shape: level out of range");
        need(valueBytes == 4 || valueBytes == 8, "b2g_level_pipe_shape: valueBytes is 4 or 8");
        const auto& pipe = mesh->m.lev[level].pipe;
        const auto it = pipe.find(nSweeps * 16 + valueBytes);
        const bool have = it != pipe.end();
        const int mode = have ? it->second.mode : 0;
        if (ranks) *ranks = mode == 1 ? it->second.sched->ranks : mode == 2 ? -it->second.items->nParts : 0;
        if (nSteps)
            *nSteps = mode == 1 ? it->second.sched->nSteps : mode == 2 ? it->second.items->maxDepth + 1 : 0;
        const bool grid = mode == 1 && it->second.sched->grid;
        if (msPipe)
            *msPipe = !have ? 0.f : mode == 2 ? it->second.msItems : grid ? it->second.msGrid : it->second.msPipe;
        if (msGrid) *msGrid = have ? it->second.msGrid : 0.f;
        if (gridForm) *gridForm = grid ? 1 : 0;
        if (msSweeps) *msSweeps = have ? it->second.msSweeps : 0.f;
        if (msShared) *msShared = have ? it->second.msPipe : 0.f;
        if (msItems) *msItems = have ? it->second.msItems : 0.f;
    });
}

b2g_status b2g_level_schedule(const b2g_mesh* mesh, int level, int* partChunkStart, int* chunkRecords)
{
    return guarded([&] {
        need(mesh != nullptr, "b2g_level_schedule: null mesh");
        need(level >= 0 && level <= mesh->m.nLevels(), "b2g_level_schedule: level out of range");
        const b2g::GsSchedule& G = mesh->m.lev[level].gs;
        cudaStream_t s = mesh->m.stream;
        if (partChunkStart && G.nParts)
            B2G_CUDA(cudaMemcpyAsync(partChunkStart, G.partChunkStart.p, sizeof(int) * (G.nParts + 1),
                                     cudaMemcpyDeviceToHost, s));
        if (chunkRecords && G.nChunks)
            B2G_CUDA(cudaMemcpyAsync(chunkRecords, G.chunkRec.p, sizeof(int) * 12 * (size_t)G.nChunks,
                                     cudaMemcpyDeviceToHost, s));
        B2G_CUDA(cudaStreamSynchronize(s));
    });
}

b2g_status b2g_level_colouring(const b2g_mesh* mesh, int level, int* nColours, int* colourStart)
{
    return guarded([&] {
        need(mesh && nColours, "b2g_level_colouring: null argument");
        need(level >= 0 && level <= mesh->m.nLevels(), "b2g_level_colouring: no such level");
        const b2g::Colouring& C = mesh->m.lev[level].mc;
        *nColours = C.nColours;
        if (colourStart)
            for (int k = 0; k <= C.nColours; ++k) colourStart[k] = C.colourStart[k];
    });
}

b2g_status b2g_level_sweep_shape(const b2g_mesh* mesh, int level, int* wholeLevelCtas, int* threadsPerBlock,
                                 float* msPerSweep)
{
    return guarded([&] {
        need(mesh && wholeLevelCtas && threadsPerBlock && msPerSweep, "b2g_level_sweep_shape: null argument");
        need(level >= 0 && level <= mesh->m.nLevels(), "b2g_level_sweep_shape: no such level");
        const b2g::Colouring& C = mesh->m.lev[level].mc;
        *wholeLevelCtas = !C.tuned ? 0 : C.cluster > 0 ? C.cluster : C.fused ? 1 : 0;
        *threadsPerBlock = C.tuned ? (C.fused || C.cluster > 0 ? 1024 : C.block) : 0;
        *msPerSweep = C.tuned ? C.msPerSweep : 0.f;
    });
}

b2g_status b2g_level_mc_pipe(const b2g_mesh* mesh, int level, int nSweeps, int symmetric, int* ranks,
                             float* msPipe, float* msColours)
{
    return guarded([&] {
        need(mesh != nullptr, "b2g_level_mc_pipe: null mesh");
        need(level >= 0 && level <= mesh->m.nLevels(), "b2g_level_mc_pipe: no such level");
        const b2g::Colouring& C = mesh->m.lev[level].mc;
        const auto it = C.pipe.find(nSweeps * 2 + (symmetric ? 1 : 0));
        const bool have = it != C.pipe.end();
        if (ranks) *ranks = have && it->second.use ? it->second.sched->ranks : 0;
        if (msPipe) *msPipe = have ? it->second.msPipe : 0.f;
        if (msColours) *msColours = have ? it->second.msColours : 0.f;
    });
}

b2g_status b2g_fold_boundary(int nCells, int nBFaces, const int32_t* faceCells, const double* internalCoeffs,
                             const double* boundaryCoeffs, const unsigned char* coupled, double* diag, double* source,
                             int memspace, void* stream)
{
    return guarded([&] {
        need(nCells > 0 && nBFaces >= 0, "b2g_fold_boundary: nCells must be positive and nBFaces non-negative");
        need(diag && source, "b2g_fold_boundary: null diag or source");
        need(nBFaces == 0 || (faceCells && internalCoeffs && boundaryCoeffs && coupled),
             "b2g_fold_boundary: null boundary array");
        need(memspace == B2G_MEM_HOST || memspace == B2G_MEM_DEVICE, "b2g_fold_boundary: bad memspace");
        cudaStream_t s = streamOf(stream);
        b2g::DBuf<int> cells, order;
        b2g::DBuf<double> ic, bc, d, src;
        b2g::DBuf<unsigned char> cp;
        stage(cells, faceCells, nBFaces, memspace, s);
        stage(ic, internalCoeffs, nBFaces, memspace, s);
        stage(bc, boundaryCoeffs, nBFaces, memspace, s);
        stage(cp, coupled, nBFaces, memspace, s);
        stage(d, static_cast<const double*>(diag), nCells, memspace, s);
        stage(src, static_cast<const double*>(source), nCells, memspace, s);
        b2g::DBuf<int> err;
        err.alloc(1, s);
        err.zero(s);
        if (nBFaces) kCheckCells<<<b2g::ceilDiv(nBFaces, 256), 256, 0, s>>>(nBFaces, nCells, cells.p, err.p);
        B2G_LAUNCH_CHECK();
        int e = 0;
        B2G_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        B2G_CUDA(cudaStreamSynchronize(s));
        need(e == 0, "b2g_fold_boundary: a face cell is outside [0, nCells)");
        // each cell's boundary faces in (patch, face) order: a stable sort of the face indices by cell
        b2g::DBuf<int> start, iota;
        b2g::DBuf<unsigned> keys;
        start.alloc(nCells + 1, s);
        b2g::countingStarts(cells.p, nBFaces, nCells, start.p, s);
        order.alloc(std::max(nBFaces, 1), s);
        iota.alloc(std::max(nBFaces, 1), s);
        keys.alloc(std::max(nBFaces, 1), s);
        if (nBFaces) kIotaInt<<<b2g::ceilDiv(nBFaces, 256), 256, 0, s>>>(nBFaces, iota.p);
        int bits = 1;
        while ((1LL << bits) < nCells) ++bits;
        b2g::sortPairs(reinterpret_cast<const unsigned*>(cells.p), keys.p, iota.p, order.p, nBFaces, bits, s);
        kFold<<<b2g::ceilDiv(nCells, 256), 256, 0, s>>>(nCells, start.p, order.p, ic.p, bc.p, cp.p, d.p, src.p);
        B2G_LAUNCH_CHECK();
        const cudaMemcpyKind back = memspace == B2G_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
        B2G_CUDA(cudaMemcpyAsync(diag, d.p, sizeof(double) * nCells, back, s));
        B2G_CUDA(cudaMemcpyAsync(source, src.p, sizeof(double) * nCells, back, s));
        B2G_CUDA(cudaStreamSynchronize(s));
    });
}

b2g_status b2g_level_scale(b2g_matrix* m, int level, double* field, double* Acf, const double* source)
{
    return guarded([&] {
        need(m && field && Acf && source, "b2g_level_scale: null argument");
        m->mat->serial = false;
        need(level >= 0 && level <= m->mat->nLevels(), "b2g_level_scale: level out of range");
        b2g::Matrix& A = *m->mat;
        A.toPos(level, static_cast<const double*>(field), A.ioBuf(0));
        A.toPos(level, source, A.ioBuf(2));
        A.scale<double>(level, A.ioBuf(0), A.ioBuf(1), A.ioBuf(2));
        A.fromPos(level, static_cast<const double*>(A.ioBuf(0)), field);
        A.fromPos(level, static_cast<const double*>(A.ioBuf(1)), Acf);
        B2G_CUDA(cudaStreamSynchronize(A.stream));
    });
}

b2g_status b2g_step_restrict(b2g_matrix* m, int step, const double* fine, double* coarse)
{
    return guarded([&] {
        need(m && fine && coarse, "b2g_step_restrict: null argument");
        need(step >= 0 && step < m->mat->nLevels(), "b2g_step_restrict: step out of range");
        b2g::Matrix& A = *m->mat;
        A.toPos(step, fine, A.ioBuf(0));
        A.restrictTo<double>(step, A.ioBuf(0), A.ioBuf(1));
        A.fromPos(step + 1, static_cast<const double*>(A.ioBuf(1)), coarse);
        B2G_CUDA(cudaStreamSynchronize(A.stream));
    });
}

b2g_status b2g_step_prolong(b2g_matrix* m, int step, const double* coarse, double* fine)
{
    return guarded([&] {
        need(m && fine && coarse, "b2g_step_prolong: null argument");
        need(step >= 0 && step < m->mat->nLevels(), "b2g_step_prolong: step out of range");
        b2g::Matrix& A = *m->mat;
        A.toPos(step + 1, coarse, A.ioBuf(0));
        A.prolongFrom<double>(step, A.ioBuf(0), A.ioBuf(1));
        A.fromPos(step, static_cast<const double*>(A.ioBuf(1)), fine);
        B2G_CUDA(cudaStreamSynchronize(A.stream));
    });
}

b2g_status b2g_level_norm_factor(b2g_matrix* m, int level, const double* psi, const double* source,
                                 const double* Apsi, double* nf)
{
    return guarded([&] {
        need(m && psi && source && Apsi && nf, "b2g_level_norm_factor: null argument");
        need(level >= 0 && level <= m->mat->nLevels(), "b2g_level_norm_factor: level out of range");
        b2g::Matrix& A = *m->mat;
        A.toPos(level, psi, A.ioBuf(0));
        A.toPos(level, source, A.ioBuf(1));
        A.toPos(level, Apsi, A.ioBuf(2));
        *nf = A.normFactor(level, A.ioBuf(0), A.ioBuf(1), A.ioBuf(2));
    });
}

b2g_status b2g_level_pcg_dic(b2g_matrix* m, int level, double* psi, const double* source, double tolerance,
                             double relTol, b2g_perf* out)
{
    return guarded([&] {
        need(m && psi && source && out, "b2g_level_pcg_dic: null argument");
        need(level >= 0 && level <= m->mat->nLevels(), "b2g_level_pcg_dic: level out of range");
        b2g::Matrix& A = *m->mat;
        const int n = A.mesh->lev[level].nCells;
        if (static_cast<int>(A.v64.cpA.n) < n)
            for (b2g::DBuf<double>* b : {&A.v64.cpA, &A.v64.cwA, &A.v64.crA, &A.v64.crD}) b->alloc(n, A.stream);
        b2g::DBuf<b2g::k::DevPerf> dp;
        dp.alloc(1, A.stream);
        A.toPos(level, static_cast<const double*>(psi), A.ioBuf(0));
        A.toPos(level, source, A.ioBuf(1));
        A.coarsestSolve<double>(level, A.ioBuf(0), A.ioBuf(1), tolerance, relTol, dp.p, false);
        A.fromPos(level, static_cast<const double*>(A.ioBuf(0)), psi);
        std::vector<b2g::k::DevPerf> h = dp.download(A.stream);
        out->initialResidual = h[0].initialResidual;
        out->finalResidual = h[0].finalResidual;
        out->nIterations = h[0].nIterations;
    });
}

b2g_status b2g_precondition(b2g_matrix* m, const b2g_controls* controls, double* w, const double* r,
                            b2g_solve_log* log)
{
    return guarded([&] {
        need(m && controls && w && r, "b2g_precondition: null argument");
        b2g::Matrix& A = *m->mat;
        need(A.nLevels() > 0, "b2g_precondition: the mesh has no coarse levels");
        A.resetLog(log ? std::max(log->coarsestCapacity, 0) : 0);
        A.serial = controls->reduction == B2G_REDUCTION_SERIAL;
        A.toPos(0, r, A.ioBuf(1));
        A.precondition(*controls, A.ioBuf(0), A.ioBuf(1));
        A.fromPos(0, static_cast<const double*>(A.ioBuf(0)), w);
        A.checkDeviceError();
        A.readLog(log);
    });
}

b2g_status b2g_matrix_pcg_solve(b2g_matrix* m, const double* source, double* psi, const b2g_controls* controls,
                                int memspace, b2g_perf* out, b2g_solve_log* log)
{
    return guarded([&] {
        need(m != nullptr, "b2g_matrix_pcg_solve: null matrix");
        b2g::capi::solveOn(*m->mat, source, psi, controls, memspace, out, log, false, false);
    });
}

b2g_status b2g_pcg_gamg_solve(b2g_mesh* mesh, const double* diag, const double* upper, const double* source,
                              double* psi, const b2g_controls* controls, int memspace, void* stream, b2g_perf* out,
                              b2g_solve_log* log)
{
    return guarded([&] {
        need(mesh && diag && controls, "b2g_pcg_gamg_solve: null argument");
        need(memspace == B2G_MEM_HOST || memspace == B2G_MEM_DEVICE, "b2g_pcg_gamg_solve: bad memspace");
        need(mesh->m.lev[0].nFaces == 0 || upper, "b2g_pcg_gamg_solve: null upper");
        (void)stream;
        if (!mesh->solveMatrix) mesh->solveMatrix.reset(new b2g::Matrix(&mesh->m, mesh->m.stream));
        b2g::Matrix& A = *mesh->solveMatrix;
        A.setFine(diag, upper, memspace);
        bool staged = false;
        if (memspace == B2G_MEM_HOST && source && psi && mesh->m.nLevels() > 0)
        {
            // the source and the initial guess cross on a second stream once the matrix has, while the
            // first builds the coarse levels (built here rather than after the first residual: the same
            // matrices, only earlier)
            b2g::capi::stageSideCopies(A, source, psi);
            A.buildCoarse();
            b2g::capi::joinSideCopies(A);
            staged = true;
        }
        b2g::capi::solveOn(A, source, psi, controls, memspace, out, log, false, staged);
    });
}

b2g_status b2g_gamg_solve(b2g_mesh* mesh, const double* diag, const double* upper, const double* source,
                          double* psi, const b2g_controls* controls, int memspace, void* stream, b2g_perf* out,
                          b2g_solve_log* log)
{
    return guarded([&] {
        need(mesh && diag && controls, "b2g_gamg_solve: null argument");
        need(memspace == B2G_MEM_HOST || memspace == B2G_MEM_DEVICE, "b2g_gamg_solve: bad memspace");
        need(mesh->m.lev[0].nFaces == 0 || upper, "b2g_gamg_solve: null upper");
        (void)stream;
        if (!mesh->solveMatrix) mesh->solveMatrix.reset(new b2g::Matrix(&mesh->m, mesh->m.stream));
        b2g::Matrix& A = *mesh->solveMatrix;
        A.setFine(diag, upper, memspace);
        b2g::capi::solveOn(A, source, psi, controls, memspace, out, log, true, false);
    });
}

b2g_status b2g_mesh_set_pair(b2g_mesh* mesh, int nPairFaces, const int32_t* faceCells, const int32_t* nbrFaceCells,
                             int memspace, void* stream)
{
    return guarded([&] {
        need(mesh && faceCells && nbrFaceCells, "b2g_mesh_set_pair: null argument");
        need(memspace == B2G_MEM_HOST || memspace == B2G_MEM_DEVICE, "b2g_mesh_set_pair: bad memspace");
        need(nPairFaces > 0, "b2g_mesh_set_pair: nPairFaces must be positive");
        (void)stream;
        std::vector<int> own(static_cast<size_t>(nPairFaces)), nbr(static_cast<size_t>(nPairFaces));
        const cudaMemcpyKind kind = memspace == B2G_MEM_HOST ? cudaMemcpyHostToHost : cudaMemcpyDeviceToHost;
        B2G_CUDA(cudaMemcpy(own.data(), faceCells, sizeof(int) * own.size(), kind));
        B2G_CUDA(cudaMemcpy(nbr.data(), nbrFaceCells, sizeof(int) * nbr.size(), kind));
        b2g::buildPair(mesh->m, nPairFaces, own.data(), nbr.data());
    });
}

b2g_status b2g_mesh_level_pair(const b2g_mesh* mesh, int level, int* nPairFaces, int32_t* own, int32_t* nbr)
{
    return guarded([&] {
        need(mesh && nPairFaces, "b2g_mesh_level_pair: null argument");
        need(level >= 0 && level <= mesh->m.nLevels(), "b2g_mesh_level_pair: level out of range");
        const b2g::PairLevel& P = mesh->m.lev[level].pair;
        *nPairFaces = P.nFaces;
        if (own) std::copy(P.own.begin(), P.own.end(), own);
        if (nbr) std::copy(P.nbr.begin(), P.nbr.end(), nbr);
    });
}

b2g_status b2g_matrix_create_coupled(b2g_mesh* mesh, const double* diag, const double* upper, const double* pairCoeffs,
                                     int memspace, void* stream, b2g_matrix** out)
{
    return guarded([&] {
        need(mesh && out && diag && pairCoeffs, "b2g_matrix_create_coupled: null argument");
        need(memspace == B2G_MEM_HOST || memspace == B2G_MEM_DEVICE, "b2g_matrix_create_coupled: bad memspace");
        need(mesh->m.lev[0].nFaces == 0 || upper, "b2g_matrix_create_coupled: null upper");
        need(mesh->m.hasPair, "b2g_matrix_create_coupled: the mesh carries no coupled pair (b2g_mesh_set_pair)");
        std::unique_ptr<b2g_matrix> h(new b2g_matrix);
        h->mesh = mesh;
        (void)stream;
        h->mat.reset(new b2g::Matrix(&mesh->m, mesh->m.stream));
        h->mat->setFine(diag, upper, memspace);
        h->mat->setPairCoeffs(pairCoeffs, memspace);
        h->mat->buildCoarse();
        B2G_CUDA(cudaStreamSynchronize(mesh->m.stream));
        *out = h.release();
    });
}

b2g_status b2g_matrix_level_pair_coeffs(const b2g_matrix* m, int level, double* coeffs)
{
    return guarded([&] {
        need(m && coeffs, "b2g_matrix_level_pair_coeffs: null argument");
        const b2g::Matrix& A = *m->mat;
        need(level >= 0 && level <= A.nLevels(), "b2g_matrix_level_pair_coeffs: level out of range");
        need(A.coupled, "b2g_matrix_level_pair_coeffs: the matrix carries no coupled pair");
        const int nF = A.mesh->lev[level].pair.nFaces;
        B2G_CUDA(cudaMemcpyAsync(coeffs, A.v64.coef[level].pairCoef.p, sizeof(double) * nF, cudaMemcpyDeviceToHost,
                                 A.stream));
        B2G_CUDA(cudaStreamSynchronize(A.stream));
    });
}

b2g_status b2g_gamg_solve_coupled(b2g_mesh* mesh, const double* diag, const double* upper, const double* pairCoeffs,
                                  const double* source, double* psi, const b2g_controls* controls, int memspace,
                                  void* stream, b2g_perf* out, b2g_solve_log* log)
{
    return guarded([&] {
        need(mesh && diag && pairCoeffs && controls, "b2g_gamg_solve_coupled: null argument");
        need(mesh->m.hasPair, "b2g_gamg_solve_coupled: the mesh carries no coupled pair (b2g_mesh_set_pair)");
        (void)stream;
        b2g::Matrix A(&mesh->m, mesh->m.stream);
        A.setFine(diag, upper, memspace);
        A.setPairCoeffs(pairCoeffs, memspace);
        b2g::capi::solveOn(A, source, psi, controls, memspace, out, log, true);
    });
}

b2g_status b2g_matrix_gamg_solve(b2g_matrix* m, const double* source, double* psi, const b2g_controls* controls,
                                 int memspace, b2g_perf* out, b2g_solve_log* log)
{
    return guarded([&] {
        need(m != nullptr, "b2g_matrix_gamg_solve: null matrix");
        b2g::capi::solveOn(*m->mat, source, psi, controls, memspace, out, log, true, false);
    });
}

b2g_status b2g_matrix_timings(const b2g_matrix* m, double* ms4, long long* counts4)
{
    return guarded([&] {
        need(m != nullptr, "b2g_matrix_timings: null matrix");
        for (int i = 0; i < 4; ++i)
        {
            if (ms4) ms4[i] = m->mat->ms[i];
            if (counts4) counts4[i] = m->mat->counts[i];
        }
    });
}

b2g_status b2g_matrix_level_timings(const b2g_matrix* m, int kind, int capacity, double* ms, long long* regions,
                                    long long* units, int* nLevels)
{
    return guarded([&] {
        need(m != nullptr, "b2g_matrix_level_timings: null matrix");
        need(kind >= 0 && kind <= 2,
             "b2g_matrix_level_timings: kind is 0 (Amul), 1 (smoothing) or 2 (Amul fused with another step)");
        const b2g::Matrix& A = *m->mat;
        const int have = static_cast<int>(A.lvMs[kind].size());
        if (nLevels) *nLevels = have;
        for (int l = 0; l < std::min(have, capacity); ++l)
        {
            if (ms) ms[l] = A.lvMs[kind][l];
            if (regions) regions[l] = A.lvCalls[kind][l];
            if (units) units[l] = A.lvUnits[kind][l];
        }
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// The coarsest-level PCG-DIC with no device allocation (b2g_level_pcg_dic_static)
// ---------------------------------------------------------------------------------------------
//
// Some callers may not allocate device memory during a solve: a host code whose device memory is
// owned by another allocator (a framework's caching pool that has reserved the GPU), or a loop that
// cannot afford the implicit device synchronisation cudaMalloc/cudaFree may bring. For them this
// entry keeps every scratch vector of the coarsest-level solve in one file-scope device array that
// the library image carries, so the call itself allocates nothing.
namespace {

constexpr int kStaticCells = 4096;  // the largest level the static scratch holds
// six vectors of kStaticCells doubles (psi and source in position order, pA, wA, rA, rD) and the
// solver-performance record: about 192 KiB, held on every GPU that loads the library until exit
constexpr size_t kStaticDoubles = 6 * static_cast<size_t>(kStaticCells) + 4;
static __device__ __align__(256) double g_staticScratch[kStaticDoubles];

// Nothing in the array needs to start at zero: each call writes every scratch value before it
// reads it (the copies of psi and source, the residual, the DIC reciprocals, the PCG vectors and
// the performance record), whatever an earlier call left there.
//
// The context current on this thread (the driver's cuCtxGetCurrent, reached through the runtime so
// that the library does not link the driver library itself), or null if it cannot be asked.
void* currentContext()
{
    using CtxGetCurrent = int (*)(void**);
    static const CtxGetCurrent fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrent>(f);
    }();
    void* ctx = nullptr;
    if (fn && fn(&ctx) != 0) ctx = nullptr;
    return ctx;
}

// The device address of g_staticScratch on the current device. In host code the symbol is only a
// host-side stand-in, so the address is looked up once per device (with that device current) and
// cached; the first call on a device does this. The cache remembers the context it was looked up
// in: after a device reset the primary context is a new one, its module a new image, and the
// address is looked up again instead of reusing the old one.
double* staticScratchAddress()
{
    struct Slot
    {
        void* ctx = nullptr;
        double* addr = nullptr;
    };
    static std::mutex mu;
    static Slot slot[64];
    int dev = 0;
    B2G_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) b2g::fail(B2G_ERR_STATE, "b2g_level_pcg_dic_static: device ordinal out of range");
    void* ctx = currentContext();
    std::lock_guard<std::mutex> lock(mu);
    if (!slot[dev].addr || slot[dev].ctx != ctx || !ctx)
    {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_staticScratch);
        if (e != cudaSuccess)
            b2g::fail(B2G_ERR_CUDA, std::string("b2g_level_pcg_dic_static: cudaGetSymbolAddress failed: ") +
                                        cudaGetErrorString(e));
        slot[dev].addr = static_cast<double*>(p);
        slot[dev].ctx = ctx;
    }
    return slot[dev].addr;
}

}  // namespace

extern "C" B2G_API b2g_status b2g_level_pcg_dic_static(b2g_matrix* m, int level, double* psi, const double* source,
                                                       double tolerance, double relTol, b2g_perf* out)
{
    return guarded([&] {
        need(m && psi && source && out, "b2g_level_pcg_dic_static: null argument");
        b2g::Matrix& A = *m->mat;
        need(level >= 0 && level <= A.nLevels(), "b2g_level_pcg_dic_static: level out of range");
        const b2g::LevelAddr& L = A.mesh->lev[level];
        const int n = L.nCells;
        if (n > kStaticCells)
            b2g::fail(B2G_ERR_ARGUMENT, "b2g_level_pcg_dic_static: the level has " + std::to_string(n) +
                                            " cells; the static scratch holds at most " +
                                            std::to_string(kStaticCells));
        int dev = 0;
        B2G_CUDA(cudaGetDevice(&dev));
        need(dev == A.mesh->device, "b2g_level_pcg_dic_static: make the matrix's device current first");
        double* base = staticScratchAddress();
        double* psiPos = base;
        double* srcPos = base + kStaticCells;
        b2g::k::DevPerf* perf = reinterpret_cast<b2g::k::DevPerf*>(base + 6 * static_cast<size_t>(kStaticCells));
        cudaStream_t s = A.stream;
        const int grid = std::max(1, (n + 255) / 256);
        if (n)
        {
            b2g::k::toPositions<double><<<grid, 256, 0, s>>>(n, L.gs.posCell.p, psi, psiPos);
            b2g::k::toPositions<double><<<grid, 256, 0, s>>>(n, L.gs.posCell.p, source, srcPos);
        }
        B2G_LAUNCH_CHECK();
        // the same kernel and arguments as b2g_level_pcg_dic, with the scratch vectors in the array
        const b2g::LevelCoef<double>& C = A.v64.coef[level];
        b2g::k::CoarsestArgs<double> a;
        a.n = n;
        a.nF = L.nFaces;
        a.lower = L.lower.p;
        a.upper = L.upper.p;
        a.posOf = L.gs.posOf.p;
        a.rowStart = L.gs.posRow.p;
        a.col = L.gs.entColPos.p;
        a.val = C.rowVal.p;
        a.diag = C.gsDiag.p;
        a.coef = C.upper.p;
        a.source = srcPos;
        a.psi = psiPos;
        a.pA = base + 2 * static_cast<size_t>(kStaticCells);
        a.wA = base + 3 * static_cast<size_t>(kStaticCells);
        a.rA = base + 4 * static_cast<size_t>(kStaticCells);
        a.rD = base + 5 * static_cast<size_t>(kStaticCells);
        a.tolerance = tolerance;
        a.relTol = relTol;
        a.maxIter = 1000;
        a.log = nullptr;
        a.logCount = nullptr;
        a.logCapacity = 0;
        a.out = perf;
        if (C.pairVal.p && L.pair.nFaces > 0)
        {
            a.pairStart = L.pair.start.p;
            a.pairCol = L.pair.col.p;
            a.pairVal = C.pairVal.p;
        }
        b2g::k::coarsestPcgDic<double><<<1, 32, 0, s>>>(a);
        B2G_LAUNCH_CHECK();
        if (n) b2g::k::fromPositions<double><<<grid, 256, 0, s>>>(n, L.gs.posCell.p, psiPos, psi);
        B2G_LAUNCH_CHECK();
        b2g::k::DevPerf h;
        B2G_CUDA(cudaMemcpyAsync(&h, perf, sizeof(h), cudaMemcpyDeviceToHost, s));
        B2G_CUDA(cudaStreamSynchronize(s));
        out->initialResidual = h.initialResidual;
        out->finalResidual = h.finalResidual;
        out->nIterations = h.nIterations;
    });
}
