// Black-box probe of how nvcc (default flags, --fmad=true) evaluates the
// reference's score expression `(double)prox + height_penalty*qz*qz*qz`
// (spectral_packing/fft3.cu:172-173).  Built by tests/test_gpu_parity.py.
#include <cuda_runtime.h>
extern "C" __global__ void score_expr(const int* prox, const int* k, int nz, double hp, double* out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        double qz = (double)k[i] / (double)nz;
        out[i] = (double)prox[i] + hp * qz * qz * qz;
    }
}
extern "C" int run_score_probe(const int* prox, const int* k, int nz, double hp, double* out, int n) {
    int *dp, *dk;
    double* dout;
    if (cudaMalloc(&dp, n * sizeof(int)) || cudaMalloc(&dk, n * sizeof(int)) || cudaMalloc(&dout, n * sizeof(double)))
        return 1;
    cudaMemcpy(dp, prox, n * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(dk, k, n * sizeof(int), cudaMemcpyHostToDevice);
    score_expr<<<(n + 255) / 256, 256>>>(dp, dk, nz, hp, dout, n);
    cudaError_t e = cudaMemcpy(out, dout, n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dp); cudaFree(dk); cudaFree(dout);
    return e != cudaSuccess;
}
