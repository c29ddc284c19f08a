// Material probes of the C ABI: Material::sample, computeBsdf and computePdf
// (src/materials/material.h:18-24) and the density / effective integrand of
// the sampling procedure, evaluated on the GPU for arrays of directions in
// the local shading frame. Compiled without FMA contraction, like the
// reference-stream integrator, so that results follow the reference's FP32
// operation order.
#include "context.cuh"

namespace {

__global__ void k_material_sample(ag::Material m, const float* wo, const float* u, uint32_t n, float* wi, float* est,
                                  float* pdf, uint8_t* ok)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ag::BsdfSample s;
    const float3 w = ag::mk3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
    const bool good = ag::mat_sample(m, w, u[2 * i], u[2 * i + 1], s);
    if (!good) s = ag::BsdfSample{ag::mk3(0.0f, 0.0f, 0.0f), ag::mk3(0.0f, 0.0f, 0.0f), 0.0f};
    wi[3 * i] = s.wi.x;
    wi[3 * i + 1] = s.wi.y;
    wi[3 * i + 2] = s.wi.z;
    est[3 * i] = s.estimator.x;
    est[3 * i + 1] = s.estimator.y;
    est[3 * i + 2] = s.estimator.z;
    pdf[i] = s.pdf;
    ok[i] = good ? 1 : 0;
}

__global__ void k_material_eval(ag::Material m, const float* wo, const float* wi, uint32_t n, float* bsdf, float* pdf,
                                float* density, float* integrand)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 a = ag::mk3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
    const float3 b = ag::mk3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
    const float3 f = ag::mat_bsdf(m, a, b);
    bsdf[3 * i] = f.x;
    bsdf[3 * i + 1] = f.y;
    bsdf[3 * i + 2] = f.z;
    pdf[i] = ag::mat_pdf(m, a, b);
    float p;
    float3 fc;
    ag::plain_eval(m, a, b, p, fc);
    density[i] = p;
    integrand[3 * i] = fc.x;
    integrand[3 * i + 1] = fc.y;
    integrand[3 * i + 2] = fc.z;
}

// Device scratch for one probe call: inputs and outputs of `n` entries.
struct Probe {
    ag::DeviceBuffer buf;
    float* at(size_t offsetFloats) { return buf.as<float>() + offsetFloats; }
};

}  // namespace

extern "C" {

int alpine_gpu_material_sample(alpine_gpu_ctx* c, const alpine_gpu_material* material, const float* wo,
                               const float* u, uint32_t n, float* wi, float* estimator, float* pdf, uint8_t* ok)
{
    if (!c || !material) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (n == 0) return ALPINE_GPU_OK;
    if (!wo || !u || !wi || !estimator || !pdf || !ok)
        return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "material_sample: null array");
    ag::Material m;
    if (!ag::make_material(*material, m)) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "material_sample: unknown kind");
    cudaSetDevice(c->device);
    const size_t N = n;
    Probe p;  // wo 3N, u 2N, wi 3N, est 3N, pdf N, ok N bytes
    if (!p.buf.reserve((12 * N) * sizeof(float) + N + 64))
        return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "material_sample: scratch");
    float *dWo = p.at(0), *dU = p.at(3 * N), *dWi = p.at(5 * N), *dEst = p.at(8 * N), *dPdf = p.at(11 * N);
    uint8_t* dOk = reinterpret_cast<uint8_t*>(p.at(12 * N));
    cudaStream_t st = c->stream;
    cudaError_t e = cudaMemcpyAsync(dWo, wo, 3 * N * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dU, u, 2 * N * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_material_sample<<<(n + 127) / 128, 128, 0, st>>>(m, dWo, dU, n, dWi, dEst, dPdf, dOk);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(wi, dWi, 3 * N * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(estimator, dEst, 3 * N * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(pdf, dPdf, N * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ok, dOk, N, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("material_sample: ") + cudaGetErrorString(e));
    return ALPINE_GPU_OK;
}

int alpine_gpu_material_eval(alpine_gpu_ctx* c, const alpine_gpu_material* material, const float* wo, const float* wi,
                             uint32_t n, float* bsdf, float* pdf, float* sample_density, float* sample_integrand)
{
    if (!c || !material) return ALPINE_GPU_ERR_INVALID_ARGUMENT;
    if (n == 0) return ALPINE_GPU_OK;
    if (!wo || !wi) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "material_eval: null array");
    ag::Material m;
    if (!ag::make_material(*material, m)) return c->fail(ALPINE_GPU_ERR_INVALID_ARGUMENT, "material_eval: unknown kind");
    cudaSetDevice(c->device);
    const size_t N = n;
    Probe p;  // wo 3N, wi 3N, bsdf 3N, pdf N, density N, integrand 3N
    if (!p.buf.reserve(14 * N * sizeof(float))) return c->fail(ALPINE_GPU_ERR_OUT_OF_MEMORY, "material_eval: scratch");
    float *dWo = p.at(0), *dWi = p.at(3 * N), *dB = p.at(6 * N), *dP = p.at(9 * N), *dD = p.at(10 * N),
          *dI = p.at(11 * N);
    cudaStream_t st = c->stream;
    cudaError_t e = cudaMemcpyAsync(dWo, wo, 3 * N * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dWi, wi, 3 * N * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_material_eval<<<(n + 127) / 128, 128, 0, st>>>(m, dWo, dWi, n, dB, dP, dD, dI);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && bsdf) e = cudaMemcpyAsync(bsdf, dB, 3 * N * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && pdf) e = cudaMemcpyAsync(pdf, dP, N * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && sample_density)
        e = cudaMemcpyAsync(sample_density, dD, N * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && sample_integrand)
        e = cudaMemcpyAsync(sample_integrand, dI, 3 * N * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return c->fail(ALPINE_GPU_ERR_CUDA, std::string("material_eval: ") + cudaGetErrorString(e));
    return ALPINE_GPU_OK;
}

}  // extern "C"
