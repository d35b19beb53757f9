// server.cu -- the serving form: a request loop for pressure solves of many independent cases.
//
// Cases are registered once: each keeps its hierarchy (the mesh handle) and its matrix (the
// Galerkin levels and every work vector) resident in HBM. Registering a case is admitted by its
// HBM footprint: idle cases are evicted, least recently used first, until the new one fits under
// the cap. Requests -- one pressure solve of a registered case, with its own source and initial
// guess -- queue as they arrive. nSlots worker threads each own a CUDA stream. A worker takes the
// oldest queued request whose case no other worker is solving, so requests that arrive while
// others are on the GPU start as soon as a slot frees up, and their work overlaps on the device.
//
// A case's sweeps keep all their parts. Sweeps of several slots may then ask for more SMs than the
// GPU has; that stays safe because a part waits only for lower-numbered parts of its own sweep
// (gs_kernels.cuh), which are dispatched first: the parts that are resident always progress and free
// their SMs, and every wait is bounded besides.
//
// A request's fields stay in the caller's buffers until its solve starts. They cross the host
// boundary through pinned staging buffers, one pair per slot (copies from pageable memory are
// synchronous and serialise across threads), and the solution goes back into the caller's psi.
//
// A solve in the mix is the same solve as alone: the same kernels on the same resident data, so
// the results are bit for bit those of b2g_matrix_pcg_solve on the case.
#include "capi_internal.cuh"

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <thread>
#include <vector>

using b2g::capi::guarded;
using b2g::capi::need;

struct b2g_server
{
    using Clock = std::chrono::steady_clock;

    struct Case
    {
        std::unique_ptr<b2g_mesh> mesh;
        std::unique_ptr<b2g::Matrix> mat;
        size_t bytes = 0;
        int nCells = 0;
        bool busy = false;
        bool alive = true;
        long long lastUse = 0;
    };
    struct Request
    {
        long long ticket = 0;
        int caseId = -1;
        const double* source = nullptr;
        double* psi = nullptr;
        size_t n = 0;
        b2g_controls controls{};
        Clock::time_point submitted;
    };
    struct Result
    {
        b2g_status status = B2G_OK;
        std::string message;
        b2g_perf perf{};
        double latencyMs = 0.0;
    };
    struct Staging
    {
        double* source = nullptr;
        double* psi = nullptr;
        size_t n = 0;
    };

    int device = 0;
    size_t capBytes = 0;
    int nSlots = 0;
    cudaStream_t buildStream = nullptr;
    std::vector<cudaStream_t> slotStreams;
    std::vector<Staging> staging;  // pinned host buffers of each slot
    std::vector<std::unique_ptr<Case>> cases;
    size_t resident = 0;
    std::deque<Request> queue;
    std::map<long long, Result> results;
    std::set<long long> outstanding;  // submitted, not yet collected by a wait
    std::mutex mu;
    std::condition_variable cvWork, cvDone;
    bool stopping = false;
    long long nextTicket = 1;
    long long useClock = 0;
    std::vector<std::thread> workers;
};

namespace {

size_t poolUsedBytes()
{
    unsigned long long used = 0;
    B2G_CUDA(cudaMemPoolGetAttribute(b2g::libraryPool(), cudaMemPoolAttrUsedMemCurrent, &used));
    return static_cast<size_t>(used);
}

// One request on one slot: the case's fields in, the PCG + GAMG (or GAMG) solve, the solution out.
void runRequest(b2g_server::Case& c, b2g_server::Request& r, cudaStream_t stream, b2g_server::Staging& st,
                b2g_server::Result& out)
{
    out.status = guarded([&] {
        b2g::Matrix& A = *c.mat;
        A.stream = stream;
        const size_t n = r.n;
        if (st.n < n)
        {
            if (st.source) B2G_CUDA(cudaFreeHost(st.source));
            if (st.psi) B2G_CUDA(cudaFreeHost(st.psi));
            st.source = st.psi = nullptr;
            st.n = 0;
            B2G_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&st.source), n * sizeof(double), cudaHostAllocDefault));
            B2G_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&st.psi), n * sizeof(double), cudaHostAllocDefault));
            st.n = n;
        }
        std::memcpy(st.source, r.source, n * sizeof(double));
        std::memcpy(st.psi, r.psi, n * sizeof(double));
        b2g::capi::solveOn(A, st.source, st.psi, &r.controls, B2G_MEM_HOST, &out.perf, nullptr,
                           r.controls.solver == B2G_SOLVER_GAMG);
        std::memcpy(r.psi, st.psi, n * sizeof(double));
    });
    if (out.status != B2G_OK) out.message = b2g::capi::lastError;
    out.latencyMs = std::chrono::duration<double, std::milli>(b2g_server::Clock::now() - r.submitted).count();
}

void workerLoop(b2g_server* S, int slot)
{
    cudaSetDevice(S->device);
    for (;;)
    {
        b2g_server::Request r;
        b2g_server::Case* c = nullptr;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            auto runnable = [&]() -> std::deque<b2g_server::Request>::iterator {
                for (auto it = S->queue.begin(); it != S->queue.end(); ++it)
                    if (!S->cases[it->caseId]->busy) return it;
                return S->queue.end();
            };
            S->cvWork.wait(lk, [&] { return S->stopping || runnable() != S->queue.end(); });
            if (S->stopping) return;
            auto it = runnable();
            r = std::move(*it);
            S->queue.erase(it);
            c = S->cases[r.caseId].get();
            c->busy = true;
            c->lastUse = ++S->useClock;
        }
        b2g_server::Result res;
        runRequest(*c, r, S->slotStreams[slot], S->staging[slot], res);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->results[r.ticket] = std::move(res);
            c->busy = false;
        }
        S->cvDone.notify_all();
        S->cvWork.notify_all();  // a request queued behind this case may run now
    }
}

// Evicts idle cases with no queued request, least recently used first, until `need` more bytes
// fit under the cap (or none is left to evict).
void evictFor(b2g_server& S, size_t need)
{
    while (S.resident + need > S.capBytes)
    {
        b2g_server::Case* victim = nullptr;
        for (size_t i = 0; i < S.cases.size(); ++i)
        {
            b2g_server::Case* c = S.cases[i].get();
            if (!c->alive || c->busy || (victim && c->lastUse >= victim->lastUse)) continue;
            bool queued = false;
            for (const auto& r : S.queue)
                if (r.caseId == static_cast<int>(i)) queued = true;
            if (!queued) victim = c;
        }
        if (!victim) return;
        victim->mat.reset();
        victim->mesh.reset();
        victim->alive = false;
        S.resident -= victim->bytes;
        victim->bytes = 0;
    }
}

}  // namespace

extern "C" {

B2G_API b2g_status b2g_server_create(unsigned long long hbmCapBytes, int nSlots, b2g_server** out)
{
    return guarded([&] {
        need(out != nullptr, "b2g_server_create: null output handle");
        need(nSlots >= 1 && nSlots <= 64, "b2g_server_create: nSlots must be in 1..64");
        need(hbmCapBytes > 0, "b2g_server_create: the HBM cap must be positive");
        std::unique_ptr<b2g_server> S(new b2g_server);
        B2G_CUDA(cudaGetDevice(&S->device));
        S->capBytes = static_cast<size_t>(hbmCapBytes);
        S->nSlots = nSlots;
        B2G_CUDA(cudaStreamCreateWithFlags(&S->buildStream, cudaStreamNonBlocking));
        S->slotStreams.resize(nSlots);
        S->staging.resize(nSlots);
        for (auto& st : S->slotStreams) B2G_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        for (int i = 0; i < nSlots; ++i) S->workers.emplace_back(workerLoop, S.get(), i);
        *out = S.release();
    });
}

B2G_API b2g_status b2g_server_destroy(b2g_server* S)
{
    return guarded([&] {
        if (!S) return;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->stopping = true;
        }
        S->cvWork.notify_all();
        for (auto& w : S->workers) w.join();
        for (auto& c : S->cases)
        {
            c->mat.reset();
            c->mesh.reset();
        }
        for (cudaStream_t st : S->slotStreams) cudaStreamSynchronize(st);
        cudaStreamSynchronize(S->buildStream);
        for (cudaStream_t st : S->slotStreams) cudaStreamDestroy(st);
        for (auto& sg : S->staging)
        {
            if (sg.source) cudaFreeHost(sg.source);
            if (sg.psi) cudaFreeHost(sg.psi);
        }
        cudaStreamDestroy(S->buildStream);
        delete S;
    });
}

B2G_API b2g_status b2g_server_add_case(b2g_server* S, int nCells, int nFaces, const int32_t* lower,
                                       const int32_t* upper, const double* Sf, const double* magSf,
                                       const double* diag, const double* upperCoef, int nCellsInCoarsestLevel,
                                       int memspace, int* caseId)
{
    return guarded([&] {
        need(S && caseId && diag, "b2g_server_add_case: null argument");
        need(nFaces == 0 || upperCoef, "b2g_server_add_case: null upper coefficients");
        int dev = 0;
        B2G_CUDA(cudaGetDevice(&dev));
        need(dev == S->device, "b2g_server_add_case: make the server's device current first");
        std::unique_ptr<b2g_server::Case> c(new b2g_server::Case);
        const size_t before = poolUsedBytes();
        int forward = 1;
        c->mesh = b2g::capi::createMesh(nCells, nFaces, lower, upper, Sf, magSf, nCellsInCoarsestLevel, &forward,
                                        memspace, S->buildStream);
        c->mat.reset(new b2g::Matrix(&c->mesh->m, S->buildStream));
        c->mat->setFine(diag, upperCoef, memspace);
        c->mat->buildCoarse();
        c->mat->ensureFp32();
        c->nCells = nCells;
        B2G_CUDA(cudaStreamSynchronize(S->buildStream));
        const size_t after = poolUsedBytes();
        c->bytes = after > before ? after - before : 0;
        std::lock_guard<std::mutex> lk(S->mu);
        // make room, else refuse: the case does not fit beside the busy or queued ones
        evictFor(*S, c->bytes);
        if (S->resident + c->bytes > S->capBytes)
            b2g::fail(B2G_ERR_NO_MEMORY, "b2g_server_add_case: the case does not fit under the HBM cap beside "
                                         "the cases in use");
        S->resident += c->bytes;
        c->lastUse = ++S->useClock;
        S->cases.push_back(std::move(c));
        *caseId = static_cast<int>(S->cases.size()) - 1;
    });
}

B2G_API b2g_status b2g_server_submit(b2g_server* S, int caseId, const double* source, double* psi,
                                     const b2g_controls* controls, long long* ticket)
{
    return guarded([&] {
        need(S && source && psi && controls && ticket, "b2g_server_submit: null argument");
        b2g_server::Request r;
        r.submitted = b2g_server::Clock::now();
        r.caseId = caseId;
        r.source = source;
        r.psi = psi;
        r.controls = *controls;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            need(caseId >= 0 && caseId < static_cast<int>(S->cases.size()) && S->cases[caseId]->alive,
                 "b2g_server_submit: no such case (never added, or evicted)");
            r.n = static_cast<size_t>(S->cases[caseId]->nCells);
            r.ticket = S->nextTicket++;
            *ticket = r.ticket;
            S->outstanding.insert(r.ticket);
            S->queue.push_back(std::move(r));
        }
        S->cvWork.notify_one();
    });
}

B2G_API b2g_status b2g_server_wait(b2g_server* S, long long ticket, b2g_perf* out, double* latencyMs, int timeoutMs)
{
    b2g_status solveStatus = B2G_OK;
    std::string solveMessage;
    const b2g_status st = guarded([&] {
        need(S != nullptr, "b2g_server_wait: null server");
        std::unique_lock<std::mutex> lk(S->mu);
        need(S->outstanding.count(ticket) != 0, "b2g_server_wait: unknown ticket, or its result was collected");
        auto ready = [&] { return S->results.count(ticket) != 0; };
        if (timeoutMs < 0) S->cvDone.wait(lk, ready);
        else if (!S->cvDone.wait_for(lk, std::chrono::milliseconds(timeoutMs), ready))
            b2g::fail(B2G_ERR_STATE, "b2g_server_wait: the request is still pending");
        b2g_server::Result res = std::move(S->results[ticket]);
        S->results.erase(ticket);
        S->outstanding.erase(ticket);
        lk.unlock();
        if (out) *out = res.perf;
        if (latencyMs) *latencyMs = res.latencyMs;
        solveStatus = res.status;
        solveMessage = res.message;
    });
    if (st != B2G_OK) return st;
    if (solveStatus != B2G_OK) b2g::capi::lastError = solveMessage;
    return solveStatus;
}

B2G_API b2g_status b2g_server_case_bytes(b2g_server* S, int caseId, unsigned long long* bytes)
{
    return guarded([&] {
        need(S && bytes, "b2g_server_case_bytes: null argument");
        std::lock_guard<std::mutex> lk(S->mu);
        need(caseId >= 0 && caseId < static_cast<int>(S->cases.size()), "b2g_server_case_bytes: no such case");
        *bytes = S->cases[caseId]->bytes;
    });
}

}  // extern "C"
