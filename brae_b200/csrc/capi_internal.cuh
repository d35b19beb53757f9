// capi_internal.cuh -- what the C-ABI translation units share: the opaque handles' definitions, the
// exception-to-status wrapper with the thread's last-error string, the mesh builder and the solve.
#pragma once

#include "solver.cuh"

#include <memory>
#include <string>

struct b2g_mesh
{
    b2g::Mesh m;
    // The matrix b2g_pcg_gamg_solve / b2g_gamg_solve solve on: kept between calls (the mesh-lifetime
    // cache of the reference's device path), its coefficients replaced by each call, so that its
    // buffers and captured iteration graphs are reused. Declared after `m`: destroyed before it.
    std::unique_ptr<b2g::Matrix> solveMatrix;
};

struct b2g_matrix
{
    b2g_mesh* mesh = nullptr;
    std::unique_ptr<b2g::Matrix> mat;
};

namespace b2g {
namespace capi {

extern thread_local std::string lastError;

// Runs f, turning the library's exceptions into status codes and the thread's last-error string.
template <class F>
b2g_status guarded(F&& f)
{
    try
    {
        f();
        return B2G_OK;
    }
    catch (const b2g::Error& e)
    {
        lastError = e.what();
        return e.code;
    }
    catch (const std::bad_alloc&)
    {
        lastError = "b2g: host allocation failed";
        return B2G_ERR_NO_MEMORY;
    }
    catch (const std::exception& e)
    {
        lastError = e.what();
        return B2G_ERR_STATE;
    }
}

// Refuses with B2G_ERR_ARGUMENT and `msg` unless `ok`.
void need(bool ok, const char* msg);

// Builds a mesh handle (the device hierarchy) on `stream` from host or device arrays. With
// `cachePath`, a cached agglomeration whose content signature matches is loaded from that file
// (*fromCache = 1), else the hierarchy is built and the file written (*fromCache = 0).
std::unique_ptr<b2g_mesh> createMesh(int nCells, int nFaces, const int32_t* lower, const int32_t* upper,
                                     const double* Sf, const double* magSf, int nCellsInCoarsestLevel,
                                     int* forwardInOut, int memspace, cudaStream_t stream,
                                     const char* cachePath = nullptr, int* fromCache = nullptr);

// A whole solve on the finest level of A (on A.stream): source and psi from `memspace`, psi
// overwritten with the solution; the PCG + GAMG solver, or GAMG alone when `standalone`.
// `staged`: host fields already copied into A.fc / A.fr (stageSideCopies, joined).
void solveOn(b2g::Matrix& A, const double* source, double* psi, const b2g_controls* c, int memspace,
             b2g_perf* out, b2g_solve_log* log, bool standalone, bool staged = false);
// Host source and psi into A.fc / A.fr on the matrix's side stream, behind the copies queued on its
// stream; joinSideCopies makes its stream wait for them.
void stageSideCopies(b2g::Matrix& A, const double* source, const double* psi);
void joinSideCopies(b2g::Matrix& A);

}  // namespace capi
}  // namespace b2g
