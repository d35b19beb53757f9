// server.cu -- the serving form: a request loop for pressure solves of many independent cases.
//
// Cases are registered once: each keeps its hierarchy (the mesh handle) and its matrix (the
// Galerkin levels and every work vector) resident in HBM. Registering a case is admitted by its
// HBM footprint: idle cases are evicted, least recently used first, until the new one fits under
// the cap. Requests -- one pressure solve of a registered case, with its own source and initial
// guess -- queue as they arrive. nSlots worker threads each own a CUDA stream and lean to one size
// class (slot i to class i mod 3). A worker takes the oldest queued request of its class whose case
// no other worker is solving (else the oldest of any class) and, with it, the queued requests of
// other idle cases of the same size class and controls (up to a class cap): the group is solved as
// ONE batch (batch.cuh), every level step one launch over all of its cases. Requests that arrive
// while others are on the GPU join the next group a slot forms, and the slots' groups overlap on
// the device. A group's batch is kept per slot (least recently used out) for the next group of the
// same cases. A case's result does not depend on the group it is solved in (per-case reductions).
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
// The standalone GAMG solver (controls->solver == B2G_SOLVER_GAMG) and the smoothers other than
// GaussSeidel are solved alone, by the single-case path (the batch sweeps GaussSeidel).
#include "batch.cuh"
#include "capi_internal.cuh"

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <algorithm>
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
        std::vector<double*> retired;  // outgrown buffers, freed with the server
    };

    int device = 0;
    size_t capBytes = 0;
    int nSlots = 0;
    cudaStream_t buildStream = nullptr;
    std::vector<cudaStream_t> slotStreams;
    std::vector<Staging> staging;  // pinned host buffers of each slot
    struct CachedBatch
    {
        std::vector<int> ids;      // the cases, ascending
        std::unique_ptr<b2g::Batch> batch;
        long long lastUse = 0;
    };
    std::vector<std::vector<CachedBatch>> batches;  // per slot
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

constexpr int kClassCells[2] = {1 << 18, 1 << 22};  // small below 262,144 cells, medium below 4,194,304
constexpr int kGroupCap[3] = {64, 16, 4};            // cases per group, by size class
constexpr size_t kBatchesPerSlot = 16;

int sizeClass(int nCells) { return nCells < kClassCells[0] ? 0 : nCells < kClassCells[1] ? 1 : 2; }

// Grows a slot's pinned buffers to at least n values, doubling. The old buffers are kept until the
// server is destroyed: cudaFreeHost waits for the whole device, which would stall every slot.
void ensureStaging(b2g_server::Staging& st, size_t n)
{
    if (st.n >= n) return;
    const size_t cap = std::max(n, 2 * st.n);
    if (st.source) st.retired.push_back(st.source);
    if (st.psi) st.retired.push_back(st.psi);
    st.source = st.psi = nullptr;
    st.n = 0;
    B2G_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&st.source), cap * sizeof(double), cudaHostAllocDefault));
    B2G_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&st.psi), cap * sizeof(double), cudaHostAllocDefault));
    st.n = cap;
}

// The standalone GAMG solve of one request.
void runAlone(b2g_server::Case& c, b2g_server::Request& r, cudaStream_t stream, b2g_server::Staging& st,
              b2g_server::Result& out)
{
    out.status = guarded([&] {
        b2g::Matrix& A = *c.mat;
        A.stream = stream;
        const size_t n = r.n;
        ensureStaging(st, n);
        std::memcpy(st.source, r.source, n * sizeof(double));
        std::memcpy(st.psi, r.psi, n * sizeof(double));
        b2g::capi::solveOn(A, st.source, st.psi, &r.controls, B2G_MEM_HOST, &out.perf, nullptr,
                           r.controls.solver == B2G_SOLVER_GAMG);
        std::memcpy(r.psi, st.psi, n * sizeof(double));
    });
    if (out.status != B2G_OK) out.message = b2g::capi::lastError;
    out.latencyMs = std::chrono::duration<double, std::milli>(b2g_server::Clock::now() - r.submitted).count();
}

// A group of requests of distinct cases as one batch; `batch` is the group's (cached) batch, its
// cases in ascending id order.
void runGroup(std::vector<b2g_server::Request>& group, b2g::Batch& batch, const std::vector<int>& ids,
              b2g_server::Staging& st, std::vector<b2g_server::Result>& out)
{
    const size_t K = group.size();
    out.assign(K, b2g_server::Result{});
    std::string message;
    const b2g_status status = guarded([&] {
        // the batch's case order: ascending ids
        std::vector<size_t> at(K);
        for (size_t i = 0; i < K; ++i)
            at[i] = static_cast<size_t>(std::lower_bound(ids.begin(), ids.end(), group[i].caseId) - ids.begin());
        std::vector<size_t> off(K + 1, 0);
        std::vector<size_t> nOf(K);
        for (size_t i = 0; i < K; ++i) nOf[at[i]] = group[i].n;
        for (size_t k = 0; k < K; ++k) off[k + 1] = off[k] + nOf[k];
        ensureStaging(st, off[K]);
        std::vector<const double*> src(K);
        std::vector<double*> psi(K);
        for (size_t i = 0; i < K; ++i)
        {
            const size_t k = at[i];
            std::memcpy(st.source + off[k], group[i].source, group[i].n * sizeof(double));
            std::memcpy(st.psi + off[k], group[i].psi, group[i].n * sizeof(double));
            src[k] = st.source + off[k];
            psi[k] = st.psi + off[k];
        }
        std::vector<b2g_perf> perfs(K);
        batch.solve(group[0].controls, src.data(), psi.data(), B2G_MEM_HOST, perfs.data());
        for (size_t i = 0; i < K; ++i)
        {
            std::memcpy(group[i].psi, st.psi + off[at[i]], group[i].n * sizeof(double));
            out[i].perf = perfs[at[i]];
        }
    });
    if (status != B2G_OK) message = b2g::capi::lastError;
    const auto now = b2g_server::Clock::now();
    for (size_t i = 0; i < K; ++i)
    {
        out[i].status = status;
        out[i].message = message;
        out[i].latencyMs = std::chrono::duration<double, std::milli>(now - group[i].submitted).count();
    }
}

void workerLoop(b2g_server* S, int slot)
{
    cudaSetDevice(S->device);
    for (;;)
    {
        std::vector<b2g_server::Request> group;
        std::vector<int> ids;
        b2g::Batch* batch = nullptr;
        bool alone = false;
        std::string buildError;
        b2g_status buildStatus = B2G_OK;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            // the oldest runnable request of this slot's size class, else the oldest of any class:
            // slots lean to one class each (small, medium, big, small, ...), so small requests do not
            // queue behind a backlog of big ones, and no slot idles while a request can run
            const int pref = slot % 3;
            auto runnable = [&]() -> std::deque<b2g_server::Request>::iterator {
                auto any = S->queue.end();
                for (auto it = S->queue.begin(); it != S->queue.end(); ++it)
                {
                    const b2g_server::Case* c = S->cases[it->caseId].get();
                    if (c->busy) continue;
                    if (sizeClass(c->nCells) == pref) return it;
                    if (any == S->queue.end()) any = it;
                }
                return any;
            };
            S->cvWork.wait(lk, [&] { return S->stopping || runnable() != S->queue.end(); });
            if (S->stopping) return;
            auto it0 = runnable();
            const b2g_controls c0 = it0->controls;
            alone = c0.solver != B2G_SOLVER_PCG_GAMG || c0.smoother != B2G_SMOOTHER_GAUSS_SEIDEL;
            const int cls = sizeClass(S->cases[it0->caseId]->nCells);
            // the oldest runnable request, then the queued requests of other idle cases that can
            // share its batch, oldest first
            bool first = true;  // it0 itself (erasing from the deque invalidates it0)
            for (auto it = it0; it != S->queue.end() && static_cast<int>(group.size()) < (alone ? 1 : kGroupCap[cls]);)
            {
                b2g_server::Case* c = S->cases[it->caseId].get();
                const bool fits = first || (!alone && !c->busy && it->controls.solver == B2G_SOLVER_PCG_GAMG &&
                                            it->controls.smoother == B2G_SMOOTHER_GAUSS_SEIDEL &&
                                            sizeClass(c->nCells) == cls &&
                                            std::memcmp(&it->controls, &c0, sizeof(b2g_controls)) == 0);
                first = false;
                if (fits)
                {
                    c->busy = true;
                    c->lastUse = ++S->useClock;
                    group.push_back(std::move(*it));
                    it = S->queue.erase(it);
                }
                else
                {
                    ++it;
                }
            }
            for (const auto& r : group) ids.push_back(r.caseId);
            std::sort(ids.begin(), ids.end());
            if (!alone)
            {
                auto& cache = S->batches[slot];
                for (auto& cb : cache)
                    if (cb.ids == ids)
                    {
                        batch = cb.batch.get();
                        cb.lastUse = ++S->useClock;
                    }
            }
        }
        std::vector<b2g_server::Result> res;
        if (alone)
        {
            res.resize(1);
            runAlone(*S->cases[group[0].caseId], group[0], S->slotStreams[slot], S->staging[slot], res[0]);
        }
        else
        {
            std::unique_ptr<b2g::Batch> made;
            if (!batch)
            {
                buildStatus = guarded([&] {
                    std::vector<b2g::Matrix*> mats;
                    for (int id : ids) mats.push_back(S->cases[id]->mat.get());
                    made.reset(new b2g::Batch(std::move(mats), S->slotStreams[slot]));
                });
                if (buildStatus != B2G_OK) buildError = b2g::capi::lastError;
                batch = made.get();
            }
            if (batch)
            {
                runGroup(group, *batch, ids, S->staging[slot], res);
            }
            else
            {
                res.assign(group.size(), b2g_server::Result{});
                for (size_t i = 0; i < group.size(); ++i)
                {
                    res[i].status = buildStatus;
                    res[i].message = buildError;
                }
            }
            if (made)
            {
                std::lock_guard<std::mutex> lk(S->mu);
                auto& cache = S->batches[slot];
                if (cache.size() >= kBatchesPerSlot)
                {
                    auto lru = std::min_element(cache.begin(), cache.end(), [](const auto& a, const auto& b) {
                        return a.lastUse < b.lastUse;
                    });
                    cache.erase(lru);
                }
                b2g_server::CachedBatch cb;
                cb.ids = ids;
                cb.batch = std::move(made);
                cb.lastUse = ++S->useClock;
                cache.push_back(std::move(cb));
            }
        }
        {
            std::lock_guard<std::mutex> lk(S->mu);
            for (size_t i = 0; i < group.size(); ++i)
            {
                S->results[group[i].ticket] = std::move(res[i]);
                S->cases[group[i].caseId]->busy = false;
            }
        }
        S->cvDone.notify_all();
        S->cvWork.notify_all();  // requests queued behind these cases may run now
    }
}

// Evicts idle cases with no queued request, least recently used first, until `need` more bytes
// fit under the cap (or none is left to evict); the cached batches that hold an evicted case go too.
void evictFor(b2g_server& S, size_t need)
{
    while (S.resident + need > S.capBytes)
    {
        b2g_server::Case* victim = nullptr;
        int victimId = -1;
        for (size_t i = 0; i < S.cases.size(); ++i)
        {
            b2g_server::Case* c = S.cases[i].get();
            if (!c->alive || c->busy || (victim && c->lastUse >= victim->lastUse)) continue;
            bool queued = false;
            for (const auto& r : S.queue)
                if (r.caseId == static_cast<int>(i)) queued = true;
            if (!queued)
            {
                victim = c;
                victimId = static_cast<int>(i);
            }
        }
        if (!victim) return;
        for (auto& cache : S.batches)
            cache.erase(std::remove_if(cache.begin(), cache.end(),
                                       [&](const b2g_server::CachedBatch& cb) {
                                           return std::binary_search(cb.ids.begin(), cb.ids.end(), victimId);
                                       }),
                        cache.end());
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
        S->batches.resize(nSlots);
        // slots that serve small cases first get the highest stream priority, big the lowest: the
        // block scheduler then starts a small group's blocks before queued blocks of long sweeps
        int least = 0, greatest = 0;
        B2G_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        for (int i = 0; i < nSlots; ++i)
        {
            const int cls = i % 3;
            const int prio = cls == 0 ? greatest : cls == 2 ? least : (least + greatest) / 2;
            B2G_CUDA(cudaStreamCreateWithPriority(&S->slotStreams[i], cudaStreamNonBlocking, prio));
        }
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
        S->batches.clear();
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
            for (double* r : sg.retired) cudaFreeHost(r);
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
