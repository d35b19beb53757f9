// solver.cuh -- one matrix on a mesh's hierarchy (GamgHierarchy) and the solves that run on it.
#pragma once

#include "coarsest_kernels.cuh"
#include "gs_kernels.cuh"
#include "hierarchy.cuh"
#include "ldu_kernels.cuh"
#include "pipe_kernels.cuh"

#include <map>

namespace b2g {

// Device-resident PCG scalars (one slot each, so a captured iteration needs no host round trip).
struct PcgScalars
{
    double wArA, wArAold, wApA, wrOld, nf, sumMag, finalRes, initRes, sumPsi;
    int singular, iter, pad0, pad1;
};

// The coefficients of one level in value type T. The LDU arrays keep the reference's cell and face
// numbering (the Galerkin sums read them); every kernel of the solve reads the position-ordered pair.
template <class T>
struct LevelCoef
{
    DBuf<T> diag;   // [nCells] by cell (FP64 only)
    DBuf<T> upper;  // [nFaces] LDU coefficient, upper == lower (FP64 only)
    DBuf<T> gsDiag; // [nCells (+pad)] diagonal by position
    DBuf<T> rowVal; // [2*nFaces] coefficient per CSR entry, rows by position
    DBuf<T> ellVal; // the same in the level's sliced ELL layout (GsSchedule::ellEnt), where it has one
    DBuf<unsigned char> blob;  // the sweep's chunk blobs (gs_kernels.cuh) in T
    DBuf<float> mcVal, mcDiag;  // FP32 only: the multicolour layout's coefficients (hierarchy.cuh Colouring)
    // FP64 only, a coupled matrix: the pair's coefficient per pair face and per row entry (pair.cu)
    DBuf<T> pairCoef, pairVal;
};

// Everything a V-cycle in value type T touches.
// Every level vector is in that level's position order and allocated to its GsSchedule::nAlloc.
template <class T>
struct VCycleData
{
    std::vector<LevelCoef<T>> coef;   // [0..nLevels]
    std::vector<DBuf<T>> corr, src;   // [coarse level index 0..nLevels-1] = mesh levels 1..nLevels
    DBuf<T> ACf, preSmoothed;         // scratch, finest size
    DBuf<T> partial;                  // reduction partials
    DBuf<T> sf;                       // scale factor slot
    DBuf<T> cpA, cwA, crA, crD;       // coarsest scratch
    // symGaussSeidel: each level's reversed layout (diagonal and chunk blobs by reversed position)
    // and the backward walk's source and psi in reversed positions
    std::vector<LevelCoef<T>> rev;
    std::vector<DBuf<T>> revB, revX;
    // DIC / DICGaussSeidel: per level the substitutions' layouts (the lower-only level's and the
    // descending reversed level's chunk blobs, diagonal 1), rD by position, and scratch vectors
    std::vector<LevelCoef<T>> dicLo, dicUp;
    std::vector<DBuf<T>> rdPos, dicR, dicLoB, dicLoX, dicUpB, dicUpX;
    // a coupled matrix: per level the Gauss-Seidel smoothers' bPrime with the pair folded in
    std::vector<DBuf<T>> pairB;
    // the coefficient generation (Matrix::coefGen) each level's reversed and DIC layouts were filled for
    std::vector<long long> revGen, dicGen;
    // item schedules (items.cu), per (level, sweeps): this matrix's chunk blobs in T, the source by
    // item, and the coefficient generation the blobs were filled for
    struct ItemBuffers
    {
        DBuf<unsigned char> blob;
        DBuf<T> b;
        long long gen = -1;
    };
    std::map<std::pair<int, int>, ItemBuffers> items;
    // FP32 form only: dense Cholesky of the coarsest level
    bool built = false;
};

// One PCG (or GAMG) iteration captured as a CUDA graph, replayed while the launches it captured stay
// valid: the key holds what they depend on beyond the matrix's fixed buffers (the controls, the
// coarsest-level log, the reduction order).
// A profiled region (b2g_set_profiling): the events around one Amul (kind 0) or one smoothing call
// (kind 1) of one level, and its units (Amuls, or the sweeps of the smoothing call).
struct TimedRegion
{
    cudaEvent_t start = nullptr, end = nullptr;
    int kind = 0, level = 0, units = 0;
};

struct IterationGraph
{
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned char> key;
    long long launchesPerReplay = 0;
    // profiling: the regions captured as event-record nodes; re-recorded by every replay, read after it
    std::vector<TimedRegion> regions;
};

// the level's rows, with the coupled pair's entries when the matrix carries one
template <class T>
k::Rows<T> rowsOf(const LevelAddr& L, const LevelCoef<T>& C)
{
    k::Rows<T> r{L.nCells, L.gs.posRow.p, L.gs.entColPos.p, C.rowVal.p, C.gsDiag.p};
    if (C.pairVal.p && L.pair.nFaces > 0)
    {
        r.pairStart = L.pair.start.p;
        r.pairCol = L.pair.col.p;
        r.pairVal = C.pairVal.p;
    }
    if (L.gs.nEllEnt && C.ellVal.p)
    {
        r.ellBase = L.gs.ellBase.p;
        r.ellCol = L.gs.ellCol.p;
        r.ellVal = C.ellVal.p;
    }
    return r;
}

// Whether smoothing calls may take the pipelined multi-sweep launch (pipe.cu; b2g_set_sweep_pipeline).
extern bool g_pipeline;
// The batched one-CTA pipelined launch (pipe.cu): n cases' levels, table = k::PipeArgs<T>[n] on the
// device, caseOf[n] each entry's case (its `active` flag; active may be null).
template <class T>
void launchPipeBatch(const void* table, const int* caseOf, int n, size_t smem, const int* active, cudaStream_t s);

struct Matrix
{
    Mesh* mesh = nullptr;
    cudaStream_t stream = nullptr;
    VCycleData<double> v64;
    VCycleData<float> v32;
    bool coarseBuilt = false;
    // finest-level work (FP64), by position
    DBuf<double> psi, source, rA, wA, pA, AwA, fc, fr, rOld;
    DBuf<double> io[4];                       // level-entry staging (b2g_level_*), finest size
    DBuf<float> r32, w32, AwA32, fc32, fr32;
    DBuf<PcgScalars> scal;
    DBuf<k::DevPerf> coarseLog;
    DBuf<int> coarseCount;
    DBuf<int> err;
    int coarseLogCapacity = 0;
    IterationGraph pcgGraph, gamgGraph;
    bool serial = false;                      // B2G_REDUCTION_SERIAL for the current solve
    // the sweep's bounded waits: polls before giving up, and whether parts publish their progress
    // (changed only by b2g_level_smooth_stall, which tests that the waits end)
    long long spinLimit = k::kSpinLimit;
    int publish = 1;
    bool coupled = false;                     // the matrix carries the mesh's coupled pair (FP64 only)
    bool multicolour = false;                 // the FP32 V-cycle sweeps colour by colour
    bool mcBuilt = false;
    // bumped by every setFine: layouts filled from the coefficients (the multicolour values, the
    // reversed and DIC layouts) are refilled, into the same buffers, when their generation is older
    long long coefGen = 0, mcGen = -1;
    std::vector<long long> rdGen;
    // timing (b2g_set_profiling): events around every level's Amuls and smoothing calls
    double ms[4] = {0, 0, 0, 0};              // finest Amul, finest smoothing, other, whole solve
    long long counts[4] = {0, 0, 0, 0};       // finest Amuls, finest sweeps, other launches, all launches
    long long launches = 0;
    std::vector<double> lvMs[3];              // per kind (0 Amul, 1 smoothing, 2 Amul fused with the residual,
                                              // the scaling or the prolongation) and level: milliseconds,
    std::vector<long long> lvCalls[3], lvUnits[3];  // timed regions, units (Amuls / sweeps)
    std::vector<TimedRegion> evOpen;          // regions recorded outside a capture, read at the end
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> evFree;
    cudaEvent_t evSolve[2] = {nullptr, nullptr};
    cudaStream_t sideStream = nullptr;        // host-field uploads beside the coarse build (capi.cu)
    cudaEvent_t sideEv[2] = {nullptr, nullptr};
    IterationGraph* capturing = nullptr;      // the graph being captured, if any
    // records a start event if profiling; the region is closed by timedEnd
    cudaEvent_t timedBegin(int kind, int level, int units);
    void timedEnd(cudaEvent_t start);
    void addRegion(const TimedRegion& r);     // a finished region into the per-level sums
    void timingsBegin();
    void timingsEnd();
    ~Matrix();

    Matrix(Mesh* m, cudaStream_t s);
    void setFine(const double* diag, const double* upper, int memspace);
    void setPairCoeffs(const double* coeff, int memspace);  // the coupled pair's coefficients (pair.cu)
    void buildCoarse();                       // Galerkin matrices of every coarse level
    void ensureFp32();                        // float copies of every level
    void ensureMulticolour();                 // the multicolour layout and its FP32 values
    void mcSmooth(int level, float* psi, const float* source, int nSweeps, bool symmetric);
    template <class T> void gsLaunch(const LevelAddr& L, const LevelCoef<T>& C, T* psi, const T* source,
                                     unsigned long long* trace, bool timed);
    template <class T> void ensureSym(int level);   // the reversed layout of `level` in T
    void prepareSmoother(const b2g_controls& c);
    std::vector<DBuf<double>> rdCell;              // DIC's reciprocal diagonal by cell, per level (FP64)
    template <class T> void ensureDic(int level);
    template <class T> void dicSmooth(int level, T* psi, const T* source, int nSweeps);
    template <class T> void symSmooth(int level, T* psi, const T* source, int nSweeps);
    void ensureResident(int level);            // the resident sweep's depth ranges (on the mesh, once)
    template <class T> bool residentSweeps(int level, T* psi, const T* source, int nSweeps);
    // the pipelined multi-sweep launch (pipe.cu): the level's tuned choice, built on first use
    template <class T> void ensurePipe(int level, int nSweeps);
    template <class T> bool pipeSweeps(int level, T* psi, const T* source, int nSweeps);
    template <class T> void pipeLaunch(int level, const PipeSchedule& P, T* psi, const T* source, bool fma = false);
    template <class T> k::PipeArgs<T> pipeArgs(int level, const PipeSchedule& P, T* psi, const T* source);
    template <class T> bool pipeForced(int level, T* psi, const T* source, int nSweeps, int ranks);
    // an item schedule's launch (items.cu): its blobs filled for the current coefficients first
    template <class T> typename VCycleData<T>::ItemBuffers& itemBuffers(int level, const GsSchedule& G);
    template <class T> void itemsLaunch(int level, const GsSchedule& G, T* psi, const T* source);
    template <class T> void refreshItems();
    // the coarsest level's dense Cholesky factor (FP32-preconditioned forms, coarsestDirect), made for
    // the current coefficients by ensureDense outside any capture
    DBuf<double> denseL;
    DBuf<int> denseOk;
    long long denseGen = -1;
    bool denseUse = false;   // the factor exists (positive definite, at most kDenseMax cells)
    bool denseNow = false;   // the current solve takes it
    void ensureDense();
    void mcLaunch(int level, bool fused, int cluster, int block, float* psi, const float* source, int nSweeps,
                  bool timed, bool symmetric = false);
    void tuneMulticolour(int level);
    // the multicolour smoothing call of nSweeps sweeps on `level` as one pipelined launch whose steps
    // are the colours (pipe.cu), chosen by timing against the tuned colour-by-colour shape; outside any
    // capture
    void ensureMcPipe(int level, int nSweeps, bool symmetric);
    int nLevels() const { return mesh->nLevels(); }
    int n(int level) const { return mesh->lev[level].nCells; }
    size_t nAlloc(int level) const { return static_cast<size_t>(std::max(mesh->lev[level].gs.nAlloc, 1)); }
    // natural cell order <-> the level's position order (device pointers)
    template <class T> void toPos(int level, const T* nat, T* pos);
    template <class T> void fromPos(int level, const T* pos, T* nat);
    double* ioBuf(int i);                     // staging vector i of the level entries

    // pieces (device pointers)
    template <class T> void amul(int level, const T* x, T* y);
    template <class T> void residualBetween(const T* source, const T* x, T* r);
    template <class T> void smooth(int level, int smoother, T* psi, const T* source, int nSweeps,
                                   unsigned long long* trace = nullptr);
    template <class T> void smoothCall(int level, int smoother, T* psi, const T* source, int nSweeps,
                                       unsigned long long* trace);
    template <class T> void scale(int level, T* field, T* Acf, const T* source);
    template <class T> void restrictTo(int step, const T* fine, T* coarse);
    template <class T> void prolongFrom(int step, const T* coarse, T* fine);
    template <class T> void coarsestSolve(int level, T* psi, const T* source, T tol, T relTol,
                                          k::DevPerf* out, bool logIt);
    template <class T> void vcycle(const b2g_controls& c, T* psi, const T* source, T* Apsi, T* fc,
                                   const T* fr);
    void precondition(const b2g_controls& c, double* w, const double* r);
    // the normalisation factor into scal->nf; read back and returned when `readBack` (else 0)
    double normFactor(int level, const double* psi, const double* source, const double* Apsi,
                      bool readBack = true);
    // sum / dot / sum of magnitudes of n values into a device slot, tree or serial per `serial`
    void reduceInto(int op, int n, const double* a, const double* b, double* slot);

    // solves on the fine level (psi/source already in this->psi/source)
    b2g_perf pcg(const b2g_controls& c, b2g_solve_log* log);
    b2g_perf gamg(const b2g_controls& c, b2g_solve_log* log);

    void resetLog(int capacity);
    void readLog(b2g_solve_log* log);
    void checkDeviceError();
    // runs `body` (the launches of one iteration) through G: captured on first use, replayed after
    template <class F> void runIteration(IterationGraph& G, const b2g_controls& c, F&& body);
    unsigned long long layoutFingerprint() const;
    void collectGraphTimings(IterationGraph& G);  // after a replay has finished
    void releaseGraph(IterationGraph& G);
    template <class T> VCycleData<T>& data();
};

}  // namespace b2g
