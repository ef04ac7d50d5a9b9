// dump.cu -- asynchronous, double-buffered field dumps.
//
// The reference writes a checkpoint by copying the whole state to the host and
// writing it with fwrite before the time loop continues (solver.cu:248-250,
// output.cu:3-44).  Here a dump costs the time loop one device-to-device
// snapshot (FP64, converted from FP32 where the state is FP32) on the solver's
// stream; the copy to pinned host memory runs on a copy stream and the files
// are written by a host thread while later steps run.  Two pinned host
// buffers: a third dump waits until the oldest one is on disk.  The files are
// the reference's raw FP64 format, `<dir>u.bin.<n>` ... `<dir>p.bin.<n>`.
//
// Memory: the device snapshot (packed state + p, FP64) and the two pinned host
// buffers are allocated by the first dump of a context and kept until the
// context is destroyed.
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>

#include "wf_internal.h"

namespace wf {

namespace {
__global__ void k_widen(double *__restrict__ dst, const float *__restrict__ src, size_t n)
{
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        dst[t] = (double)src[t];
}
}  // namespace

struct Dumper {
    int device = 0;
    Parameters layout;        // Nx, Ny, Nz, Nz_Y_max for the file writer
    size_t S = 0, N = 0;      // packed state and pressure sizes (values)
    double *d_stage = nullptr;
    double *h[2] = {nullptr, nullptr};
    cudaStream_t cs = nullptr;
    cudaEvent_t staged = nullptr, d2h[2] = {nullptr, nullptr};
    bool d2h_pending = false;   // a copy out of d_stage may still run
    int next = 0;

    struct Job {
        int buf, n;
        std::string dir;
    };
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Job> jobs;
    bool busy[2] = {false, false};
    bool stop = false;
    wf_status err = WF_OK;
    std::string err_msg;
    std::thread writer;

    void run()
    {
        cudaSetDevice(device);
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !jobs.empty(); });
                if (jobs.empty()) return;
                j = jobs.front();
                jobs.pop_front();
            }
            wf_status st = WF_OK;
            std::string msg;
            const cudaError_t e = cudaEventSynchronize(d2h[j.buf]);
            if (e != cudaSuccess) {
                st = WF_ERR_CUDA;
                msg = std::string("dump: copy to host failed: ") + cudaGetErrorString(e);
            } else {
                st = wf_save_fields(&layout, j.dir.c_str(), j.n, h[j.buf], h[j.buf] + S);
                if (st) msg = wf_last_error();
            }
            std::lock_guard<std::mutex> lk(mu);
            if (st && !err) {
                err = st;
                err_msg = msg;
            }
            busy[j.buf] = false;
            cv.notify_all();
        }
    }
};

Dumper *dumper_create(int device, const Parameters &P, size_t S, size_t N)
{
    Dumper *d = new Dumper;
    d->device = device;
    d->layout = P;
    d->S = S;
    d->N = N;
    return d;
}

// Releases what a failed set-up allocated, so that a later dump tries again.
static void dumper_release(Dumper *d)
{
    for (int b = 0; b < 2; b++) {
        if (d->d2h[b]) cudaEventDestroy(d->d2h[b]);
        if (d->h[b]) cudaFreeHost(d->h[b]);
        d->d2h[b] = nullptr;
        d->h[b] = nullptr;
    }
    if (d->staged) cudaEventDestroy(d->staged);
    if (d->cs) cudaStreamDestroy(d->cs);
    if (d->d_stage) cudaFree(d->d_stage);
    d->staged = nullptr;
    d->cs = nullptr;
    d->d_stage = nullptr;
    cudaGetLastError();
}

static wf_status dumper_setup(Dumper *d)
{
    const size_t bytes = sizeof(double) * (d->S + d->N);
    bool ok = cudaMalloc(&d->d_stage, bytes) == cudaSuccess;
    if (!ok) {
        dumper_release(d);
        set_error("dump: device snapshot of %zu bytes could not be allocated", bytes);
        return WF_ERR_OOM;
    }
    for (int b = 0; b < 2 && ok; b++) ok = cudaHostAlloc((void **)&d->h[b], bytes, cudaHostAllocDefault) == cudaSuccess;
    if (!ok) {
        dumper_release(d);
        set_error("dump: pinned host buffer of %zu bytes could not be allocated", bytes);
        return WF_ERR_OOM;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&d->cs, cudaStreamNonBlocking);
    if (!e) e = cudaEventCreateWithFlags(&d->staged, cudaEventDisableTiming);
    for (int b = 0; b < 2 && !e; b++) e = cudaEventCreateWithFlags(&d->d2h[b], cudaEventDisableTiming);
    if (e) {
        dumper_release(d);
        set_error("dump: stream or event creation failed: %s", cudaGetErrorString(e));
        return WF_ERR_CUDA;
    }
    d->writer = std::thread([d] { d->run(); });
    return WF_OK;
}

// Device side of one dump into host buffer b (snapshot, then copy to host).
static cudaError_t dumper_copy(Dumper *d, cudaStream_t s, const void *state, bool fp32, const double *p, int b)
{
    cudaError_t e = cudaSuccess;
    // the previous dump's copy must have left the snapshot before it is rewritten
    if (d->d2h_pending) e = cudaStreamWaitEvent(s, d->d2h[1 - b], 0);
    if (!e) {
        if (fp32) {
            k_widen<<<592, 256, 0, s>>>(d->d_stage, (const float *)state, d->S);
            e = cudaGetLastError();
        } else {
            e = cudaMemcpyAsync(d->d_stage, state, sizeof(double) * d->S, cudaMemcpyDeviceToDevice, s);
        }
    }
    if (!e) e = cudaMemcpyAsync(d->d_stage + d->S, p, sizeof(double) * d->N, cudaMemcpyDeviceToDevice, s);
    if (!e) e = cudaEventRecord(d->staged, s);
    if (!e) e = cudaStreamWaitEvent(d->cs, d->staged, 0);
    if (!e) e = cudaMemcpyAsync(d->h[b], d->d_stage, sizeof(double) * (d->S + d->N), cudaMemcpyDeviceToHost, d->cs);
    if (!e) e = cudaEventRecord(d->d2h[b], d->cs);
    return e;
}

wf_status dumper_enqueue(Dumper *d, cudaStream_t s, const void *state, bool fp32, const double *p, const char *dir,
                         int n)
{
    if (!d->d_stage) {
        const wf_status st = dumper_setup(d);
        if (st) return st;
    }
    int b;
    {
        std::unique_lock<std::mutex> lk(d->mu);
        b = d->next;
        d->cv.wait(lk, [&] { return !d->busy[b]; });   // back-pressure: that buffer's files are written
        d->busy[b] = true;
        d->next = 1 - b;
    }
    const cudaError_t e = dumper_copy(d, s, state, fp32, p, b);
    if (e) {
        {
            std::lock_guard<std::mutex> lk(d->mu);
            d->busy[b] = false;   // nothing will write this buffer: free it again
        }
        d->cv.notify_all();
        set_error("dump: %s", cudaGetErrorString(e));
        return WF_ERR_CUDA;
    }
    d->d2h_pending = true;
    {
        std::lock_guard<std::mutex> lk(d->mu);
        d->jobs.push_back(Dumper::Job{b, n, std::string(dir)});
    }
    d->cv.notify_all();
    return WF_OK;
}

wf_status dumper_wait(Dumper *d)
{
    if (!d) return WF_OK;
    std::unique_lock<std::mutex> lk(d->mu);
    d->cv.wait(lk, [&] { return d->jobs.empty() && !d->busy[0] && !d->busy[1]; });
    const wf_status st = d->err;
    if (st) set_error("%s", d->err_msg.c_str());
    d->err = WF_OK;
    d->err_msg.clear();
    return st;
}

void dumper_destroy(Dumper *d)
{
    if (!d) return;
    if (d->writer.joinable()) {
        dumper_wait(d);
        {
            std::lock_guard<std::mutex> lk(d->mu);
            d->stop = true;
        }
        d->cv.notify_all();
        d->writer.join();
    }
    if (d->cs) cudaStreamSynchronize(d->cs);
    dumper_release(d);
    delete d;
}

}  // namespace wf
