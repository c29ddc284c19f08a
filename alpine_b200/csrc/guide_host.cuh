// Host-side interface of the learned guide (parameters, inference, training).
#pragma once

#include "guide.cuh"

namespace ag {
namespace guide {

class Guide {
public:
    Guide() = default;
    ~Guide();
    Guide(const Guide&) = delete;
    Guide& operator=(const Guide&) = delete;

    // (Re)initialises all parameters deterministically from `seed`.
    int reset(uint32_t seed, cudaStream_t st);
    bool ready() const { return ready_; }
    void set_scene_box(float3 lo, float3 hi);
    Params params() const;
    // raw: n x 40 fp32 mixture parameters.
    // status (optional): device word that receives kErrTensorWait bits.
    void infer(const Query* q, uint32_t n, float* raw, cudaStream_t st, uint32_t* status = nullptr) const;
    // The same for a queue whose length (at most maxN) is in device memory;
    // with `packed`, out receives the decoded mixtures that the shading
    // kernel samples instead of the raw parameters: kPacked field arrays of
    // maxN floats (field f of query i at out[f * maxN + i]).
    void infer_queue(const Query* q, const uint32_t* count, uint32_t maxN, float* out, cudaStream_t st,
                     uint32_t* status = nullptr, bool packed = false) const;
    // Inference kernel: warp-level mma.sync tiles of 32 queries, or tcgen05
    // MMAs with tensor-memory accumulators on tiles of 128 queries.
    static constexpr int kKernelWarpMma = 0, kKernelTensorMemory = 1;
    void set_kernel(int k) { kernel_ = k; }
    int kernel() const { return kernel_; }
    // Adds the gradient of the batch s[offset + i * stride], i < n (mean
    // loss, scaled by invBatch) to the gradient buffers, without an update.
    void accumulate_gradients(const Sample* s, uint32_t n, float invBatch, cudaStream_t st, uint32_t offset = 0,
                              uint32_t stride = 1, uint32_t* status = nullptr);
    // Weight-gradient kernel (dW = dY^T X per layer): warp-level mma.sync
    // tiles, or tcgen05 MMAs with tensor-memory accumulators.
    void set_gradient_kernel(int k) { gradKernel_ = k; }
    int gradient_kernel() const { return gradKernel_; }
    void apply_adam(float lr, cudaStream_t st);
    // gradients + Adam; returns the batch loss (synchronises).
    float train_step(const Sample* s, uint32_t n, float lr, cudaStream_t st);
    // Sum of the batch losses of the gradient passes since reset_loss.
    void reset_loss(cudaStream_t st) { cudaMemsetAsync(loss_, 0, 4, st); }
    void read_loss_async(float* hostPinned, cudaStream_t st) const
    {
        cudaMemcpyAsync(hostPinned, loss_, 4, cudaMemcpyDeviceToHost, st);
    }
    // Recomputes the BF16 / FP16 compute copies from the FP32 masters.
    void publish(cudaStream_t st);

    float* weight_master() const { return wP_; }
    float* weight_grad() const { return wG_; }
    float* grid_master() const { return gridP_; }
    float* grid_grad() const { return gridG_; }
    uint32_t steps() const { return step_; }

private:
    bool allocate();
    void release();

    void* mem_ = nullptr;
    bool ready_ = false;
    int kernel_ = kKernelWarpMma;
    int gradKernel_ = kKernelTensorMemory;
    uint32_t step_ = 0;
    float* gridP_ = nullptr;
    float* gridM_ = nullptr;
    float* gridV_ = nullptr;
    float* gridG_ = nullptr;
    __half* gridH_ = nullptr;
    float* wP_ = nullptr;
    float* wM_ = nullptr;
    float* wV_ = nullptr;
    float* wG_ = nullptr;
    __nv_bfloat16* wB_ = nullptr;
    __nv_bfloat16* wT_ = nullptr;
    float* partial_ = nullptr;   // per-split weight gradients
    __nv_bfloat16* xt_ = nullptr;  // layer inputs of a training slice, transposed
    __nv_bfloat16* dt_ = nullptr;  // layer output gradients of a training slice, transposed
    float* loss_ = nullptr;
    float3 bmin_ = make_float3(0.0f, 0.0f, 0.0f);
    float3 invExtent_ = make_float3(1.0f, 1.0f, 1.0f);
};

}  // namespace guide
}  // namespace ag
