// solver.cuh -- one matrix on a mesh's hierarchy (GamgHierarchy) and the solves that run on it.
#pragma once

#include "coarsest_kernels.cuh"
#include "gs_kernels.cuh"
#include "hierarchy.cuh"
#include "ldu_kernels.cuh"

namespace b2g {

// Device-resident PCG scalars (one slot each, so a captured iteration needs no host round trip).
struct PcgScalars
{
    double wArA, wArAold, wApA, wrOld, nf, sumMag, finalRes, initRes, sumPsi;
    int singular, iter, pad0, pad1;
};

// The coefficient layout of one level in value type T.
template <class T>
struct LevelCoef
{
    DBuf<T> diag;   // [nCells]
    DBuf<T> upper;  // [nFaces] LDU coefficient (upper == lower)
    DBuf<T> val;    // [2*nFaces] row-layout coefficient
};

// Everything a V-cycle in value type T touches.
template <class T>
struct VCycleData
{
    std::vector<LevelCoef<T>> coef;   // [0..nLevels]
    std::vector<DBuf<T>> corr, src;   // [coarse level index 0..nLevels-1] = mesh levels 1..nLevels
    DBuf<T> ACf, preSmoothed;         // scratch, finest size
    DBuf<T> partial;                  // reduction partials
    DBuf<T> sf;                       // scale factor slot
    DBuf<T> cpA, cwA, crA, crD;       // coarsest scratch
    // FP32 form only: dense Cholesky of the coarsest level
    bool built = false;
};

struct Matrix
{
    Mesh* mesh = nullptr;
    cudaStream_t stream = nullptr;
    VCycleData<double> v64;
    VCycleData<float> v32;
    bool coarseBuilt = false;
    // finest-level work (FP64)
    DBuf<double> psi, source, rA, wA, pA, AwA, fc, fr, rOld;
    DBuf<float> r32, w32, AwA32, fc32, fr32;
    DBuf<PcgScalars> scal;
    DBuf<k::DevPerf> coarseLog;
    DBuf<int> coarseCount;
    DBuf<int> err;
    int coarseLogCapacity = 0;
    // timing
    double ms[4] = {0, 0, 0, 0};
    long long launches = 0;

    Matrix(Mesh* m, cudaStream_t s);
    void setFine(const double* diag, const double* upper, int memspace);
    void buildCoarse();                       // Galerkin matrices of every coarse level
    void ensureFp32();                        // float copies of every level
    int nLevels() const { return mesh->nLevels(); }
    int n(int level) const { return mesh->lev[level].nCells; }

    // pieces (device pointers)
    template <class T> void amul(int level, const T* x, T* y);
    template <class T> void smooth(int level, int smoother, T* psi, const T* source, int nSweeps);
    template <class T> void scale(int level, T* field, T* Acf, const T* source);
    template <class T> void restrictTo(int step, const T* fine, T* coarse);
    template <class T> void prolongFrom(int step, const T* coarse, T* fine);
    template <class T> void coarsestSolve(int level, T* psi, const T* source, T tol, T relTol,
                                          k::DevPerf* out, bool logIt);
    template <class T> void vcycle(const b2g_controls& c, T* psi, const T* source, T* Apsi, T* fc,
                                   const T* fr);
    void precondition(const b2g_controls& c, double* w, const double* r);
    double normFactor(int level, const double* psi, const double* source, const double* Apsi);

    // solves on the fine level (psi/source already in this->psi/source)
    b2g_perf pcg(const b2g_controls& c, b2g_solve_log* log);
    b2g_perf gamg(const b2g_controls& c, b2g_solve_log* log);

    void resetLog(int capacity);
    void readLog(b2g_solve_log* log);
    void checkDeviceError();
    template <class T> VCycleData<T>& data();
};

}  // namespace b2g
