// Asynchronous exchange of whole fields between host and device, for callers that keep the model
// state on the host and hand it to the library every step (the reference's own arrays, a coupler).
//
// The synchronous atjup_gpu_upload / atjup_gpu_download copy on the compute stream and wait, so a
// step that exchanges its state costs its copies plus its compute. Here the copies run on two
// copy streams of their own: an upload lands in a device staging buffer while the previous step
// still computes, atjup_gpu_apply_uploads makes the staged fields live in the compute stream's
// order, and a download snapshots the field in the compute stream's order (a device-to-device
// copy) and copies the snapshot to the host on the second copy stream while the next step
// computes. The staging buffers are double-buffered by round (one round = the uploads applied by
// one atjup_gpu_apply_uploads and the downloads after it), and each buffer has an event recorded
// after its last reader, which the next writer of that buffer waits for. A device with PCIe in
// both directions then overlaps upload, compute and download of consecutive steps.
#include "ctx.cuh"

namespace atjup {
namespace {

int xfer_init(AtjupCtx* c) {
    if (c->xfer_on) return ATJUP_OK;
    ATJUP_CUDA(cudaStreamCreateWithFlags(&c->x_h2d, cudaStreamNonBlocking));
    ATJUP_CUDA(cudaStreamCreateWithFlags(&c->x_d2h, cudaStreamNonBlocking));
    for (int s = 0; s < 2; s++) {
        ATJUP_CUDA(cudaEventCreateWithFlags(&c->x_up_done[s], cudaEventDisableTiming));
        for (int q = 0; q < ATJUP_F_COUNT; q++) {
            ATJUP_CUDA(cudaEventCreateWithFlags(&c->x_up_free[s][q], cudaEventDisableTiming));
            ATJUP_CUDA(cudaEventCreateWithFlags(&c->x_out_free[s][q], cudaEventDisableTiming));
        }
    }
    ATJUP_CUDA(cudaEventCreateWithFlags(&c->x_out_ready, cudaEventDisableTiming));
    c->xfer_on = true;
    return ATJUP_OK;
}

// both rounds' staging buffers of a field (pair[0], pair[1]) are allocated at its first exchange,
// so a steady exchange allocates nothing (a cudaMalloc in a later round would wait for the device)
int stage_buffer(AtjupCtx* c, double** pair0, double** pair1) {
    const AtjupParams& P = c->P;
    for (double** p : {pair0, pair1})
        if (!*p) ATJUP_CUDA(cudaMalloc(p, sizeof(double) * (size_t)P.im * P.jm * P.km));
    return ATJUP_OK;
}

}  // namespace

void xfer_free(AtjupCtx* c) {
    if (!c->xfer_on) return;
    cudaStreamSynchronize(c->x_h2d);
    cudaStreamSynchronize(c->x_d2h);
    for (int s = 0; s < 2; s++)
        for (int q = 0; q < ATJUP_F_COUNT; q++) {
            cudaFree(c->x_up[s][q]);
            cudaFree(c->x_out[s][q]);
            c->x_up[s][q] = c->x_out[s][q] = nullptr;
        }
    for (int s = 0; s < 2; s++) {
        cudaEventDestroy(c->x_up_done[s]);
        for (int q = 0; q < ATJUP_F_COUNT; q++) {
            cudaEventDestroy(c->x_up_free[s][q]);
            cudaEventDestroy(c->x_out_free[s][q]);
        }
    }
    cudaEventDestroy(c->x_out_ready);
    cudaStreamDestroy(c->x_h2d);
    cudaStreamDestroy(c->x_d2h);
    c->xfer_on = false;
}

int xfer_synchronize(AtjupCtx* c) {
    if (!c->xfer_on) return ATJUP_OK;
    ATJUP_CUDA(cudaStreamSynchronize(c->x_h2d));
    ATJUP_CUDA(cudaStreamSynchronize(c->x_d2h));
    return ATJUP_OK;
}

}  // namespace atjup

using namespace atjup;

extern "C" {

int atjup_gpu_upload_async(AtjupCtx* c, int32_t id, const double* host) {
    if (!c || !host || id < 0 || id >= ATJUP_F_COUNT) { set_error("upload_async: bad argument"); return ATJUP_ERR_ARG; }
    int rc = xfer_init(c);
    if (rc) return rc;
    const int s = c->x_round & 1;
    if ((rc = stage_buffer(c, &c->x_up[0][id], &c->x_up[1][id]))) return rc;
    // the buffer's last reader (the apply of the round before last) must be done with it
    ATJUP_CUDA(cudaStreamWaitEvent(c->x_h2d, c->x_up_free[s][id], 0));
    const AtjupParams& P = c->P;
    ATJUP_CUDA(cudaMemcpyAsync(c->x_up[s][id], host, sizeof(double) * (size_t)P.im * P.jm * P.km,
                               cudaMemcpyHostToDevice, c->x_h2d));
    c->x_pending[s] |= 1ull << id;
    return ATJUP_OK;
}

int atjup_gpu_apply_uploads(AtjupCtx* c) {
    if (!c) { set_error("apply_uploads: null context"); return ATJUP_ERR_ARG; }
    int rc = xfer_init(c);
    if (rc) return rc;
    const int s = c->x_round & 1;
    if (c->x_pending[s]) {
        ATJUP_CUDA(cudaEventRecord(c->x_up_done[s], c->x_h2d));
        ATJUP_CUDA(cudaStreamWaitEvent(c->stream, c->x_up_done[s], 0));
        for (int id = 0; id < ATJUP_F_COUNT; id++)
            if (c->x_pending[s] >> id & 1ull) {
                if ((rc = launch_pad(c, c->x_up[s][id], c->f[id]))) return rc;
                ATJUP_CUDA(cudaEventRecord(c->x_up_free[s][id], c->stream));
            }
        c->x_pending[s] = 0;
    }
    c->x_round++;
    return ATJUP_OK;
}

int atjup_gpu_download_async(AtjupCtx* c, int32_t id, double* host) {
    if (!c || !host || id < 0 || id >= ATJUP_F_COUNT) { set_error("download_async: bad argument"); return ATJUP_ERR_ARG; }
    int rc = xfer_init(c);
    if (rc) return rc;
    const int s = c->x_round & 1;
    if ((rc = stage_buffer(c, &c->x_out[0][id], &c->x_out[1][id]))) return rc;
    // the buffer's last reader (an earlier copy to the host) must be done with it
    ATJUP_CUDA(cudaStreamWaitEvent(c->stream, c->x_out_free[s][id], 0));
    if ((rc = launch_unpad(c, c->f[id], c->x_out[s][id]))) return rc;
    ATJUP_CUDA(cudaEventRecord(c->x_out_ready, c->stream));
    ATJUP_CUDA(cudaStreamWaitEvent(c->x_d2h, c->x_out_ready, 0));
    const AtjupParams& P = c->P;
    ATJUP_CUDA(cudaMemcpyAsync(host, c->x_out[s][id], sizeof(double) * (size_t)P.im * P.jm * P.km,
                               cudaMemcpyDeviceToHost, c->x_d2h));
    ATJUP_CUDA(cudaEventRecord(c->x_out_free[s][id], c->x_d2h));
    return ATJUP_OK;
}

}  // extern "C"
