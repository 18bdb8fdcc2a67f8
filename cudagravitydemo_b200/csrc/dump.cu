// dump.cu — the reference's outputDump.bin, written from device state.
//
// Format (basicGravity.cu:614-635, inputOutput.c:41-58): int32 body count,
// int32 frame count, RGB (3 x uint8) per body, then per frame float32 x, y, z
// per body.  The reference orders each frame by the sort's last permutation
// with a host qsort (and that permutation is not cumulative, so its frames
// are not in a fixed body order).  Here a kernel scatters every body's
// position to its slot by body id, the copy to pinned host memory is
// asynchronous, and the file write of frame k happens while the GPU steps
// towards frame k + 1 (two host buffers).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bh_internal.cuh"

__global__ void k_dump_gather(const float4* __restrict__ pos, const uint32_t* __restrict__ ids, int n,
                              float3* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = pos[i];
        const uint32_t id = ids ? ids[i] : (uint32_t)i;
        if (id < (uint32_t)n) out[id] = make_float3(p.x, p.y, p.z);
    }
}

struct bh_dump {
    FILE* f;
    int n, frames, written, enqueued;
    float3* staging;     // device, n
    float3* host[2];     // pinned, n each
    cudaEvent_t ready[2];
};

static int dump_write(bh_dump* d, int slot) {
    cudaError_t e = cudaEventSynchronize(d->ready[slot]);
    if (e != cudaSuccess) return bh_note_cuda_error(e);
    if (fwrite(d->host[slot], sizeof(float3), (size_t)d->n, d->f) != (size_t)d->n) return BH_ERR_INVALID;
    d->written++;
    return BH_OK;
}

static void dump_free(bh_dump* d) {
    if (!d) return;
    if (d->f) fclose(d->f);
    if (d->staging) cudaFree(d->staging);
    for (int k = 0; k < 2; k++) {
        if (d->host[k]) cudaFreeHost(d->host[k]);
        if (d->ready[k]) cudaEventDestroy(d->ready[k]);
    }
    free(d);
}

extern "C" int bh_dump_open(bh_dump** out, const char* path, int n, int frames, const RGB* colours) {
    if (!out || !path || n <= 0 || frames < 0) return BH_ERR_INVALID;
    *out = nullptr;
    bh_dump* d = (bh_dump*)calloc(1, sizeof(bh_dump));
    if (!d) return BH_ERR_ALLOC;
    d->n = n;
    d->frames = frames;
    cudaError_t e = cudaMalloc(&d->staging, sizeof(float3) * n);
    for (int k = 0; k < 2 && e == cudaSuccess; k++) {
        e = cudaMallocHost(&d->host[k], sizeof(float3) * n);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&d->ready[k], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        dump_free(d);
        return bh_note_cuda_error(e);
    }
    d->f = fopen(path, "wb");
    if (!d->f) {
        dump_free(d);
        return BH_ERR_INVALID;
    }
    int head[2] = {n, frames};
    bool ok = fwrite(head, sizeof(int), 2, d->f) == 2;
    RGB grey = {100, 100, 100};  // the reference's constant colour (basicGravity.cu:631-634)
    for (int i = 0; i < n && ok; i++) ok = fwrite(colours ? &colours[i] : &grey, sizeof(RGB), 1, d->f) == 1;
    if (!ok) {
        dump_free(d);
        return BH_ERR_INVALID;
    }
    *out = d;
    return BH_OK;
}

extern "C" int bh_dump_frame(bh_dump* d, const float4* pos, const uint32_t* ids, int n, cudaStream_t s) {
    if (!d || !pos || n != d->n) return BH_ERR_INVALID;
    if (d->enqueued >= d->frames) return BH_ERR_INVALID;  // more frames than the header announced
    const int slot = d->enqueued & 1;
    const int blocks = (n + 255) / 256 < 4 * bh_sm_count() ? (n + 255) / 256 : 4 * bh_sm_count();
    k_dump_gather<<<blocks, 256, 0, s>>>(pos, ids, n, d->staging);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(d->host[slot], d->staging, sizeof(float3) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaEventRecord(d->ready[slot], s);
    if (e != cudaSuccess) return bh_note_cuda_error(e);
    d->enqueued++;
    // the previous frame's copy was enqueued before this one: write it now,
    // while the device works on what the caller enqueued since
    if (d->enqueued >= 2) return dump_write(d, slot ^ 1);
    return BH_OK;
}

extern "C" int bh_sim_dump_frame(bh_dump* d, bh_sim* sim) {
    float4* pos = nullptr;
    uint32_t* ids = nullptr;
    int n = 0;
    int rc = bh_sim_device_state(sim, &pos, nullptr, &ids, &n);
    if (rc) return rc;
    return bh_dump_frame(d, pos, ids, n, bh_sim_stream(sim));
}

extern "C" int bh_dump_close(bh_dump* d) {
    if (!d) return BH_ERR_INVALID;
    int rc = BH_OK;
    if (d->enqueued > d->written) rc = dump_write(d, (d->enqueued - 1) & 1);
    if (rc == BH_OK && d->written != d->frames) rc = BH_ERR_INVALID;  // fewer frames than announced
    if (d->f && fclose(d->f) != 0 && rc == BH_OK) rc = BH_ERR_INVALID;
    d->f = nullptr;
    dump_free(d);
    return rc;
}
