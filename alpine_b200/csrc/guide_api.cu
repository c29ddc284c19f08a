// C ABI of the learned guide: parameter access, inference and training on
// host buffers (tests, tools), used by the integrator through the context.
#include "context.cuh"
#include "guide_host.cuh"

#include <cstring>
#include <vector>

using ag::DeviceBuffer;
namespace G = ag::guide;

namespace {

int ensure_guide(alpine_gpu_ctx* c)
{
    if (c->guide.ready()) return ALPINE_GPU_OK;
    if (c->guide.reset(c->guideSeed, c->stream) != 0)
        return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "guide: parameter allocation failed");
    return ALPINE_GPU_OK;
}

__global__ void k_sample_mixture(const float* raw, const float* u, uint32_t n, float* dirs, float* pdfs)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // the packed form the shading kernel samples
    float r[40], lobes[G::kPacked];
    for (int k = 0; k < 40; ++k) r[k] = raw[k];
    G::pack_mixture(r, lobes, 1);
    float3 d = G::lobes_sample(lobes, 1, u[3 * i], u[3 * i + 1], u[3 * i + 2]);
    dirs[3 * i] = d.x;
    dirs[3 * i + 1] = d.y;
    dirs[3 * i + 2] = d.z;
    pdfs[i] = G::lobes_pdf(lobes, 1, d);
}

__global__ void k_gather(const float* src, const uint64_t* idx, uint32_t n, float* dst)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}

__global__ void k_scatter(float* dst, const uint64_t* idx, uint32_t n, const float* src)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[idx[i]] = src[i];
}

}  // namespace

extern "C" {

int alpine_gpu_guide_dims(uint32_t* weight_count, uint64_t* grid_params, uint32_t* table_size, uint32_t* resolutions)
{
    if (weight_count) *weight_count = G::kWeightCount;
    if (grid_params) *grid_params = G::kGridParams;
    if (table_size) *table_size = G::kTableSize;
    if (resolutions) {
        G::Guide tmp;
        G::Params p = tmp.params();
        for (int l = 0; l < G::kLevels; ++l) resolutions[l] = p.res[l];
    }
    return ALPINE_GPU_OK;
}

int alpine_gpu_guide_reset(alpine_gpu_ctx* c, uint32_t seed, const float lo[3], const float hi[3])
{
    if (!c || !lo || !hi) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    c->guideSeed = seed;
    c->guideLastLossSteps = 0;
    if (c->guide.reset(seed, c->stream) != 0) return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "guide: reset failed");
    c->guide.set_scene_box(make_float3(lo[0], lo[1], lo[2]), make_float3(hi[0], hi[1], hi[2]));
    c->guideBoxSet = true;
    return ALPINE_GPU_OK;
}

int alpine_gpu_guide_steps(alpine_gpu_ctx* c, uint32_t* adam_steps, uint32_t* guided_waves, float* last_loss)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (adam_steps) *adam_steps = c->guide.steps();
    if (guided_waves) *guided_waves = c->guideWaveIndex;
    if (last_loss) {
        // hStatus[2] is written by the render's last training pass, complete
        // once the render has synchronised
        float sum;
        std::memcpy(&sum, c->hStatus + 2, sizeof(float));
        *last_loss = c->guideLastLossSteps ? sum / (float)c->guideLastLossSteps : 0.0f;
    }
    return ALPINE_GPU_OK;
}

int alpine_gpu_guide_infer(alpine_gpu_ctx* c, const float* queries, uint32_t n, float* raw)
{
    if (!c || (n && (!queries || !raw))) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (int rc = ensure_guide(c)) return rc;
    DeviceBuffer dq, dr;
    if (!dq.reserve((size_t)n * sizeof(G::Query)) || !dr.reserve((size_t)n * 40 * 4))
        return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "guide_infer buffers");
    cudaError_t e = cudaMemcpyAsync(dq.ptr, queries, (size_t)n * sizeof(G::Query), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        c->guide.infer(dq.as<G::Query>(), n, dr.as<float>(), c->stream, c->dStatus);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(raw, dr.ptr, (size_t)n * 40 * 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("guide_infer: ") + cudaGetErrorString(e));
    return c->check_device_status();
}

int alpine_gpu_guide_infer_device(alpine_gpu_ctx* c, const float* queries, uint32_t n, float* raw, void* stream)
{
    if (!c || (n && (!queries || !raw))) return c ? c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "null buffer") : -1;
    if (int rc = ensure_guide(c)) return rc;
    if (n == 0) return ALPINE_GPU_OK;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    c->guide.infer(reinterpret_cast<const G::Query*>(queries), n, raw, st, c->dStatus);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("guide_infer_device: ") + cudaGetErrorString(e));
    return ALPINE_GPU_OK;
}

int alpine_gpu_guide_set_gradient_kernel(alpine_gpu_ctx* c, int kernel)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (kernel == ALPINE_GPU_GUIDE_KERNEL_WARP_MMA) c->guide.set_gradient_kernel(G::Guide::kKernelWarpMma);
    else if (kernel == ALPINE_GPU_GUIDE_KERNEL_TENSOR_MEMORY) c->guide.set_gradient_kernel(G::Guide::kKernelTensorMemory);
    else return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "guide_set_gradient_kernel: unknown kernel");
    return ALPINE_GPU_OK;
}

int alpine_gpu_guide_set_kernel(alpine_gpu_ctx* c, int kernel)
{
    if (!c) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (kernel == ALPINE_GPU_GUIDE_KERNEL_WARP_MMA) c->guide.set_kernel(G::Guide::kKernelWarpMma);
    else if (kernel == ALPINE_GPU_GUIDE_KERNEL_TENSOR_MEMORY) c->guide.set_kernel(G::Guide::kKernelTensorMemory);
    else return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "guide_set_kernel: unknown kernel");
    return ALPINE_GPU_OK;
}

// Gradient of the mean loss over the batch (no update): dW (all weights,
// fp32) and, at the requested grid parameter indices, the grid gradient.
int alpine_gpu_guide_gradients(alpine_gpu_ctx* c, const float* samples, uint32_t n, float* dW,
                               const uint64_t* grid_index, uint32_t grid_count, float* grid_grad, float* loss)
{
    if (!c || (n && !samples)) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (int rc = ensure_guide(c)) return rc;
    DeviceBuffer ds, di, dg;
    if (!ds.reserve((size_t)n * sizeof(G::Sample)) || !di.reserve((size_t)grid_count * 8 + 8) ||
        !dg.reserve((size_t)grid_count * 4 + 4))
        return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "guide_gradients buffers");
    cudaStream_t st = c->stream;
    cudaError_t e = cudaMemcpyAsync(ds.ptr, samples, (size_t)n * sizeof(G::Sample), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->guide.weight_grad(), 0, G::kWeightCount * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->guide.grid_grad(), 0, G::kGridParams * 4, st);
    if (e == cudaSuccess) {
        c->guide.accumulate_gradients(ds.as<G::Sample>(), n, n ? 1.0f / (float)n : 0.0f, st, 0, 1, c->dStatus);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && dW) e = cudaMemcpyAsync(dW, c->guide.weight_grad(), G::kWeightCount * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && grid_count && grid_index && grid_grad) {
        e = cudaMemcpyAsync(di.ptr, grid_index, (size_t)grid_count * 8, cudaMemcpyHostToDevice, st);
        k_gather<<<(grid_count + 255) / 256, 256, 0, st>>>(c->guide.grid_grad(), di.as<uint64_t>(), grid_count, dg.as<float>());
        if (e == cudaSuccess) e = cudaMemcpyAsync(grid_grad, dg.ptr, (size_t)grid_count * 4, cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    // leave clean gradient buffers behind
    cudaMemsetAsync(c->guide.weight_grad(), 0, G::kWeightCount * 4, st);
    cudaMemsetAsync(c->guide.grid_grad(), 0, G::kGridParams * 4, st);
    cudaStreamSynchronize(st);
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("guide_gradients: ") + cudaGetErrorString(e));
    (void)loss;
    return ALPINE_GPU_OK;
}

int alpine_gpu_guide_train(alpine_gpu_ctx* c, const float* samples, uint32_t n, float lr, float* loss)
{
    if (!c || (n && !samples)) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (int rc = ensure_guide(c)) return rc;
    DeviceBuffer ds;
    if (!ds.reserve((size_t)n * sizeof(G::Sample))) return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "guide_train buffer");
    cudaError_t e = cudaMemcpyAsync(ds.ptr, samples, (size_t)n * sizeof(G::Sample), cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, "guide_train upload");
    float l = c->guide.train_step(ds.as<G::Sample>(), n, lr, c->stream);
    e = cudaGetLastError();
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("guide_train: ") + cudaGetErrorString(e));
    if (loss) *loss = l;
    return ALPINE_GPU_OK;
}

int alpine_gpu_guide_get_weights(alpine_gpu_ctx* c, float* w)
{
    if (!c || !w) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (int rc = ensure_guide(c)) return rc;
    if (cudaMemcpy(w, c->guide.weight_master(), G::kWeightCount * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return c->fail(ALPINE_GPU_ERR_CUDA, "guide_get_weights");
    return ALPINE_GPU_OK;
}

int alpine_gpu_guide_set_weights(alpine_gpu_ctx* c, const float* w)
{
    if (!c || !w) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (int rc = ensure_guide(c)) return rc;
    if (cudaMemcpy(c->guide.weight_master(), w, G::kWeightCount * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        return c->fail(ALPINE_GPU_ERR_CUDA, "guide_set_weights");
    c->guide.publish(c->stream);
    cudaStreamSynchronize(c->stream);
    return ALPINE_GPU_OK;
}

// Reads / writes grid parameters (fp32 masters) at flat indices
// ((level * table_size + entry) * 2 + feature).
int alpine_gpu_guide_grid(alpine_gpu_ctx* c, const uint64_t* index, uint32_t n, float* read, const float* write)
{
    if (!c || (n && !index)) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (int rc = ensure_guide(c)) return rc;
    for (uint32_t i = 0; i < n; ++i)
        if (index[i] >= G::kGridParams) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "guide_grid: index out of range");
    DeviceBuffer di, dv;
    if (!di.reserve((size_t)n * 8 + 8) || !dv.reserve((size_t)n * 4 + 4))
        return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "guide_grid buffers");
    cudaStream_t st = c->stream;
    cudaError_t e = cudaMemcpyAsync(di.ptr, index, (size_t)n * 8, cudaMemcpyHostToDevice, st);
    if (write && e == cudaSuccess) {
        e = cudaMemcpyAsync(dv.ptr, write, (size_t)n * 4, cudaMemcpyHostToDevice, st);
        k_scatter<<<(n + 255) / 256, 256, 0, st>>>(c->guide.grid_master(), di.as<uint64_t>(), n, dv.as<float>());
        c->guide.publish(st);
    }
    if (read && e == cudaSuccess) {
        k_gather<<<(n + 255) / 256, 256, 0, st>>>(c->guide.grid_master(), di.as<uint64_t>(), n, dv.as<float>());
        e = cudaMemcpyAsync(read, dv.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("guide_grid: ") + cudaGetErrorString(e));
    return ALPINE_GPU_OK;
}

// Samples n directions from the mixture given by 40 raw parameters
// (u: 3 uniform numbers per sample) and returns the mixture pdf of each.
int alpine_gpu_guide_sample_mixture(alpine_gpu_ctx* c, const float* raw, const float* u, uint32_t n, float* dirs,
                                    float* pdfs)
{
    if (!c || !raw || (n && (!u || !dirs || !pdfs))) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    DeviceBuffer dr, du, dd, dp;
    if (!dr.reserve(160) || !du.reserve((size_t)n * 12 + 4) || !dd.reserve((size_t)n * 12 + 4) ||
        !dp.reserve((size_t)n * 4 + 4))
        return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "sample_mixture buffers");
    cudaStream_t st = c->stream;
    cudaError_t e = cudaMemcpyAsync(dr.ptr, raw, 160, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(du.ptr, u, (size_t)n * 12, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && n) k_sample_mixture<<<(n + 255) / 256, 256, 0, st>>>(dr.as<float>(), du.as<float>(), n, dd.as<float>(), dp.as<float>());
    if (e == cudaSuccess) e = cudaMemcpyAsync(dirs, dd.ptr, (size_t)n * 12, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(pdfs, dp.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("sample_mixture: ") + cudaGetErrorString(e));
    return ALPINE_GPU_OK;
}

}  // extern "C"
