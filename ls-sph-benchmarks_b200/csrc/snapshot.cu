// snapshot.cu -- data/<step>.dat snapshots (write_data_mod.f90:22-56) that do not stop the
// time loop.  The synchronous lssph_write_data downloads the state and writes the file
// before returning; lssph_write_data_async only enqueues work:
//   1. on the solve's stream, device-to-device copies of x, y, u, v, rho, pre (, tem) into a
//      snapshot slot (a few microseconds; later steps may then overwrite the state);
//   2. on a side stream, after (1): one copy of the slot to pinned host memory, then a host
//      callback that writes the file in the reference's layout.
// Two slots alternate, so a snapshot can be in flight while the next is captured.  A slot's
// device buffer is reused only after its previous host copy is done (the solve's stream
// waits on that event; the copy is long finished when snapshots are a few steps apart), and
// its host buffer only after the previous file write (both run on the side stream).  Write
// errors are kept and returned by the next async call or by lssph_snapshot_wait.

#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "handle.h"

namespace lssph {

struct SnapSlot {
    double* dev = nullptr;    // kFields * N doubles
    double* host = nullptr;   // pinned, same layout
    cudaEvent_t captured = nullptr, copied = nullptr;
    bool used = false;
};

struct SnapState {
    static constexpr int kFields = 7;   // x, y, u, v, rho, pre, tem
    cudaStream_t side = nullptr;
    SnapSlot slot[2];
    int next = 0;
    size_t n = 0;
    bool tem = false;
    std::vector<int32_t> ptype;
    std::mutex mu;
    int err = LSSPH_OK;
    std::string msg;
};

namespace {

struct WriteJob {
    SnapState* s;
    const double* host;
    std::string path;
};

// Host callback on the side stream: no CUDA calls here.
void CUDART_CB write_job(void* arg) {
    WriteJob* j = static_cast<WriteJob*>(arg);
    SnapState* s = j->s;
    const size_t n = s->n;
    const double* b = j->host;
    std::string msg;
    const int rc = write_data_file(j->path, (int)n, s->tem, s->ptype.data(), b, b + n, b + 2 * n, b + 3 * n, b + 4 * n,
                                   b + 5 * n, s->tem ? b + 6 * n : nullptr, &msg);
    if (rc != LSSPH_OK) {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->err == LSSPH_OK) {
            s->err = rc;
            s->msg = msg;
        }
    }
    delete j;
}

int sfail(lssph_handle* h, int code, const std::string& msg) {
    h->err = msg;
    set_last_error(msg);
    return code;
}

int init_state(lssph_handle* h) {
    SnapState* s = new SnapState();
    h->snap = s;
    s->n = (size_t)h->num_total;
    s->tem = h->has_tem;
    s->ptype = h->ptype;
    const size_t bytes = sizeof(double) * SnapState::kFields * s->n;
    if (cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking) != cudaSuccess) return LSSPH_E_CUDA;
    for (SnapSlot& sl : s->slot) {
        if (cudaMalloc((void**)&sl.dev, bytes) != cudaSuccess) return LSSPH_E_CUDA;
        if (cudaMallocHost((void**)&sl.host, bytes) != cudaSuccess) return LSSPH_E_CUDA;
        if (cudaEventCreateWithFlags(&sl.captured, cudaEventDisableTiming) != cudaSuccess) return LSSPH_E_CUDA;
        if (cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming) != cudaSuccess) return LSSPH_E_CUDA;
    }
    return LSSPH_OK;
}

int take_error(lssph_handle* h) {
    SnapState* s = h->snap;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->err == LSSPH_OK) return LSSPH_OK;
    const int rc = s->err;
    h->err = "snapshot: " + s->msg;
    set_last_error(h->err);
    s->err = LSSPH_OK;
    s->msg.clear();
    return rc;
}

}  // namespace

// Wait for every snapshot of h and free the snapshot state (handle teardown).
void snapshot_release(lssph_handle* h) {
    SnapState* s = h->snap;
    if (!s) return;
    if (s->side) cudaStreamSynchronize(s->side);
    for (SnapSlot& sl : s->slot) {
        if (sl.dev) cudaFree(sl.dev);
        if (sl.host) cudaFreeHost(sl.host);
        if (sl.captured) cudaEventDestroy(sl.captured);
        if (sl.copied) cudaEventDestroy(sl.copied);
    }
    if (s->side) cudaStreamDestroy(s->side);
    delete s;
    h->snap = nullptr;
}

}  // namespace lssph

using namespace lssph;

extern "C" {

int lssph_write_data_async(lssph_handle* h, const char* results_root, int32_t step) {
    if (!h || !results_root) return set_last_error("null argument"), LSSPH_E_BAD_PARAM;
    if (!h->snap) {
        const int rc = init_state(h);
        if (rc != LSSPH_OK) {
            snapshot_release(h);
            return sfail(h, rc, "lssph_write_data_async: cannot set up the snapshot buffers");
        }
    }
    int rc = take_error(h);
    if (rc != LSSPH_OK) return rc;
    SnapState* s = h->snap;
    const std::string dir = std::string(results_root) + "/" + h->p.save_name + "/data";
    if (make_dirs(dir) != LSSPH_OK) return sfail(h, LSSPH_E_IO, "cannot create " + dir);
    SnapSlot& sl = s->slot[s->next];
    s->next ^= 1;
    const size_t n = s->n, bytes = sizeof(double) * n;
    const Fld& F = h->F[h->sb];
    cudaError_t e = cudaSuccess;
    if (sl.used) e = cudaStreamWaitEvent(h->stream, sl.copied, 0);   // device buffer free again
    const double* src[SnapState::kFields] = {F.x, F.y, F.u, F.v, F.rho, F.pre, h->has_tem ? F.tem : nullptr};
    for (int k = 0; k < SnapState::kFields && e == cudaSuccess; ++k)
        if (src[k]) e = cudaMemcpyAsync(sl.dev + k * n, src[k], bytes, cudaMemcpyDeviceToDevice, h->stream);
    if (e == cudaSuccess) e = cudaEventRecord(sl.captured, h->stream);
    // a batch steps its members on its own stream: make the capture complete before the
    // next batch call can touch the state
    if (e == cudaSuccess && h->batch) e = cudaEventSynchronize(sl.captured);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s->side, sl.captured, 0);
    const size_t all = (size_t)(h->has_tem ? 7 : 6) * bytes;
    if (e == cudaSuccess) e = cudaMemcpyAsync(sl.host, sl.dev, all, cudaMemcpyDeviceToHost, s->side);
    if (e == cudaSuccess) e = cudaEventRecord(sl.copied, s->side);
    if (e == cudaSuccess) {
        WriteJob* j = new WriteJob{s, sl.host, dir + "/" + std::to_string(step) + ".dat"};
        e = cudaLaunchHostFunc(s->side, write_job, j);
        if (e != cudaSuccess) delete j;
    }
    if (e != cudaSuccess) return sfail(h, LSSPH_E_CUDA, std::string("lssph_write_data_async: ") + cudaGetErrorString(e));
    sl.used = true;
    return LSSPH_OK;
}

int lssph_snapshot_wait(lssph_handle* h) {
    if (!h) return set_last_error("null handle"), LSSPH_E_BAD_PARAM;
    if (!h->snap) return LSSPH_OK;
    const cudaError_t e = cudaStreamSynchronize(h->snap->side);
    if (e != cudaSuccess) return sfail(h, LSSPH_E_CUDA, std::string("lssph_snapshot_wait: ") + cudaGetErrorString(e));
    return take_error(h);
}

}  // extern "C"
