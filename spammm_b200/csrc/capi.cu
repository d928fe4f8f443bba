// capi.cu -- library-wide C ABI pieces: error text, ABI version and the FP32
// peak probe used as the denominator of the grid-build roofline.
#include "spm_internal.cuh"
#include <cstring>

namespace spm {

static thread_local char g_last_error[1024] = {0};

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

void clear_error() { g_last_error[0] = 0; }

namespace {

constexpr int PROBE_CHAINS = 8;

// PROBE_CHAINS independent FFMA chains per thread; FLOPs = 2 * chains * iters.
__global__ void __launch_bounds__(256) fp32_probe_kernel(int iters, float seed, float* sink) {
    float a[PROBE_CHAINS];
#pragma unroll
    for (int c = 0; c < PROBE_CHAINS; c++) a[c] = seed + (float)(threadIdx.x + c);
    const float m = 0.999999f, b = 1e-7f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int c = 0; c < PROBE_CHAINS; c++) a[c] = fmaf(a[c], m, b);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < PROBE_CHAINS; c++) s += a[c];
    if (s == 1234.5678f) sink[0] = s;  // never true for this seed: keeps the chains live
}

// Same with packed fma.rn.f32x2 (two FP32 FMAs per instruction); FLOPs = 4 * chains * iters.
__global__ void __launch_bounds__(256) fp32x2_probe_kernel(int iters, float seed, float* sink) {
    unsigned long long a[PROBE_CHAINS];
#pragma unroll
    for (int c = 0; c < PROBE_CHAINS; c++) {
        const float lo = seed + (float)(threadIdx.x + c), hi = lo + 0.5f;
        asm("mov.b64 %0, {%1, %2};" : "=l"(a[c]) : "f"(lo), "f"(hi));
    }
    unsigned long long m, b;
    asm("mov.b64 %0, {%1, %1};" : "=l"(m) : "f"(0.999999f));
    asm("mov.b64 %0, {%1, %1};" : "=l"(b) : "f"(1e-7f));
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int c = 0; c < PROBE_CHAINS; c++) asm("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(a[c]) : "l"(m), "l"(b));
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < PROBE_CHAINS; c++) {
        float lo, hi;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a[c]));
        s += lo + hi;
    }
    if (s == 1234.5678f) sink[0] = s;
}

}  // namespace
}  // namespace spm

extern "C" int spm_abi_version(void) { return SPM_ABI_VERSION; }

extern "C" const char* spm_last_error(void) { return spm::g_last_error; }

extern "C" int spm_fp32_peak_probe(int iters, double* out_flops, void* stream) {
    using namespace spm;
    clear_error();
    SPM_REQUIRE(iters > 0 && out_flops, "spm_fp32_peak_probe: iters must be > 0 and out_flops non-null");
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return set_error(SPM_ERR_CUDA, "spm_fp32_peak_probe: cannot query the device");
    cudaStream_t st = as_stream(stream);
    const int blocks = sms * 8, threads = 256;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.0;
    cudaError_t err = cudaSuccess;
    for (int variant = 0; variant < 2 && err == cudaSuccess; variant++) {
        float ms = 0.f;
        for (int rep = 0; rep < 2 && err == cudaSuccess; rep++) {  // rep 0 warms up
            cudaEventRecord(e0, st);
            if (variant == 0) fp32_probe_kernel<<<blocks, threads, 0, st>>>(iters, 1.0f, nullptr);
            else fp32x2_probe_kernel<<<blocks, threads, 0, st>>>(iters, 1.0f, nullptr);
            cudaEventRecord(e1, st);
            err = cudaEventSynchronize(e1);
            if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        }
        if (err == cudaSuccess) {
            const double flops = (variant == 0 ? 2.0 : 4.0) * PROBE_CHAINS * (double)iters * blocks * threads;
            best = fmax(best, flops / (ms * 1e-3));
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err != cudaSuccess) return set_error(SPM_ERR_CUDA, "spm_fp32_peak_probe: %s", cudaGetErrorString(err));
    *out_flops = best;  // the higher of the scalar FFMA and packed FFMA2 rates
    return SPM_OK;
}
