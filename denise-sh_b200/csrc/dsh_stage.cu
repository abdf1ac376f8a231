/*
 * dsh_stage.cu — asynchronous staging of observed data for the shot loop.
 *
 * The reference reads each shot's observed traces from SU files right before
 * its residual (inseis, src/denise.c:1364-1420), so the file system and the
 * computation take turns.  A stager reads the files of queued batches on a
 * host thread into page-locked buffers (dsh_read_su, identical values) and
 * copies a batch to the device on its own stream when the caller acquires
 * it; the caller's stream waits for that copy through an event, and the
 * buffer is reused once the caller's stream has passed dsh_stager_release.
 * Batch i uses slot i % nbuf; the reader starts batch i once batch i - nbuf
 * is released and its host-to-device copy is complete.
 */
#include "dsh.h"
#include "dsh_io.h"

#include <cuda_runtime.h>

#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

struct Job {
    std::vector<std::string> paths;
    std::vector<int> ntr;
    int ns = 0;
    long long nfloats = 0;
    int status = DSH_OK;
    bool ready = false;
};

struct Slot {
    float *host = nullptr;
    float *dev = nullptr;
    bool pinned = false;
    cudaEvent_t copied = nullptr;     /* recorded on the copy stream after the upload */
    cudaEvent_t done = nullptr;       /* recorded on the caller's stream at release */
    bool copy_pending = false;
};

}  // namespace

struct dsh_stager {
    int nbuf = 0;
    long long cap = 0;
    bool device = false;
    int dev_id = 0;
    cudaStream_t copy_st = nullptr;
    std::vector<Slot> slots;
    std::deque<Job> jobs;             /* jobs[k] is batch base + k */
    long long base = 0;               /* index of jobs.front() */
    long long submitted = 0, acquired = 0, released = 0, read_next = 0;
    std::mutex mu;
    std::condition_variable cv;
    bool stop = false;
    std::thread worker;
};

static Job *job_at(dsh_stager *s, long long i) { return &s->jobs[(size_t)(i - s->base)]; }

static void reader(dsh_stager *s)
{
    if (s->device) cudaSetDevice(s->dev_id);
    for (;;) {
        long long i;
        Job job;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            /* batch i may start when it is queued and batch i - nbuf is released */
            s->cv.wait(lk, [&] { return s->stop || (s->read_next < s->submitted && s->released > s->read_next - s->nbuf); });
            if (s->stop) return;
            i = s->read_next;
            Job *j = job_at(s, i);
            job.paths = j->paths; job.ntr = j->ntr; job.ns = j->ns;
        }
        Slot &sl = s->slots[(size_t)(i % s->nbuf)];
        if (sl.copy_pending) {                         /* the previous upload from this host buffer */
            cudaEventSynchronize(sl.copied);
            sl.copy_pending = false;
        }
        int st = DSH_OK;
        long long off = 0;
        for (size_t k = 0; k < job.paths.size() && st == DSH_OK; k++) {
            if (dsh_read_su(job.paths[k].c_str(), job.ntr[k], job.ns, sl.host + off) != DSH_OK) st = DSH_ERR_PARAM;
            off += (long long)job.ntr[k] * job.ns;
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            Job *j = job_at(s, i);
            j->status = st;
            j->ready = true;
            s->read_next = i + 1;
        }
        s->cv.notify_all();
    }
}

extern "C" dsh_stager *dsh_stager_create(int nbuf, long long max_floats, int use_device, int *status)
{
    auto fail = [&](int code, dsh_stager *s) -> dsh_stager * {
        if (status) *status = code;
        if (s) dsh_stager_destroy(s);
        return nullptr;
    };
    if (nbuf < 1 || nbuf > 16 || max_floats < 1) return fail(DSH_ERR_PARAM, nullptr);
    dsh_stager *s = new dsh_stager();
    s->nbuf = nbuf;
    s->cap = max_floats;
    s->device = use_device != 0;
    s->slots.resize((size_t)nbuf);
    const size_t bytes = (size_t)max_floats * sizeof(float);
    if (s->device) {
        if (cudaGetDevice(&s->dev_id) != cudaSuccess) return fail(DSH_ERR_CUDA, s);
        if (cudaStreamCreateWithFlags(&s->copy_st, cudaStreamNonBlocking) != cudaSuccess) return fail(DSH_ERR_CUDA, s);
    }
    for (Slot &sl : s->slots) {
        if (s->device) {
            if (cudaMallocHost(&sl.host, bytes) != cudaSuccess) return fail(DSH_ERR_OOM, s);
            sl.pinned = true;
            if (cudaMalloc(&sl.dev, bytes) != cudaSuccess) return fail(DSH_ERR_OOM, s);
            if (cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess)
                return fail(DSH_ERR_CUDA, s);
        } else {
            sl.host = static_cast<float *>(malloc(bytes));
            if (!sl.host) return fail(DSH_ERR_OOM, s);
        }
    }
    s->worker = std::thread(reader, s);
    if (status) *status = DSH_OK;
    return s;
}

extern "C" int dsh_stager_submit(dsh_stager *s, int nfiles, const char *const *paths, const int *ntr, int ns)
{
    if (!s || nfiles < 1 || !paths || !ntr || ns < 1) return DSH_ERR_PARAM;
    Job j;
    for (int k = 0; k < nfiles; k++) {
        if (!paths[k] || ntr[k] < 0) return DSH_ERR_PARAM;
        j.paths.emplace_back(paths[k]);
        j.ntr.push_back(ntr[k]);
        j.nfloats += (long long)ntr[k] * ns;
    }
    j.ns = ns;
    if (j.nfloats > s->cap) return DSH_ERR_PARAM;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->jobs.push_back(std::move(j));
        s->submitted++;
    }
    s->cv.notify_all();
    return DSH_OK;
}

/* waits until the oldest unacquired batch is read; returns its index or -1 */
static long long wait_ready(dsh_stager *s)
{
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->acquired >= s->submitted || s->acquired > s->released + s->nbuf - 1) return -1;
    const long long i = s->acquired;
    s->cv.wait(lk, [&] { return job_at(s, i)->ready; });
    return i;
}

extern "C" int dsh_stager_acquire(dsh_stager *s, void *stream, const float **dev, long long *nfloats)
{
    if (!s || !s->device || !dev) return DSH_ERR_PARAM;
    if (s->acquired > s->released) return DSH_ERR_STATE;      /* one batch at a time */
    const long long i = wait_ready(s);
    if (i < 0) return DSH_ERR_STATE;
    Slot &sl = s->slots[(size_t)(i % s->nbuf)];
    int st;
    long long n;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        st = job_at(s, i)->status;
        n = job_at(s, i)->nfloats;
    }
    if (cudaSetDevice(s->dev_id) != cudaSuccess) return DSH_ERR_CUDA;
    /* the caller's previous use of this device buffer, then the upload */
    if (cudaStreamWaitEvent(s->copy_st, sl.done, 0) != cudaSuccess ||
        cudaMemcpyAsync(sl.dev, sl.host, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, s->copy_st) != cudaSuccess ||
        cudaEventRecord(sl.copied, s->copy_st) != cudaSuccess ||
        cudaStreamWaitEvent((cudaStream_t)stream, sl.copied, 0) != cudaSuccess)
        return DSH_ERR_CUDA;
    sl.copy_pending = true;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->acquired = i + 1;
    }
    *dev = sl.dev;
    if (nfloats) *nfloats = n;
    return st;
}

extern "C" int dsh_stager_acquire_host(dsh_stager *s, const float **host, long long *nfloats)
{
    if (!s || s->device || !host) return DSH_ERR_PARAM;
    if (s->acquired > s->released) return DSH_ERR_STATE;
    const long long i = wait_ready(s);
    if (i < 0) return DSH_ERR_STATE;
    int st;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        st = job_at(s, i)->status;
        if (nfloats) *nfloats = job_at(s, i)->nfloats;
        s->acquired = i + 1;
    }
    *host = s->slots[(size_t)(i % s->nbuf)].host;
    return st;
}

extern "C" int dsh_stager_release(dsh_stager *s, void *stream)
{
    if (!s) return DSH_ERR_PARAM;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->released >= s->acquired) return DSH_ERR_STATE;
        const long long i = s->released;
        if (s->device && cudaEventRecord(s->slots[(size_t)(i % s->nbuf)].done, (cudaStream_t)stream) != cudaSuccess)
            return DSH_ERR_CUDA;
        s->released = i + 1;
        while (s->base < s->released && s->base < s->read_next) {   /* drop finished jobs */
            s->jobs.pop_front();
            s->base++;
        }
    }
    s->cv.notify_all();
    return DSH_OK;
}

extern "C" int dsh_stager_destroy(dsh_stager *s)
{
    if (!s) return DSH_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    if (s->copy_st) cudaStreamSynchronize(s->copy_st);
    for (Slot &sl : s->slots) {
        if (sl.pinned) cudaFreeHost(sl.host);
        else free(sl.host);
        if (sl.dev) cudaFree(sl.dev);
        if (sl.copied) cudaEventDestroy(sl.copied);
        if (sl.done) cudaEventDestroy(sl.done);
    }
    if (s->copy_st) cudaStreamDestroy(s->copy_st);
    delete s;
    return DSH_OK;
}
