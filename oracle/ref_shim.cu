// ref_shim.cu — TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference CUDA library from its own source file, where it
// lies, into oracle/_ref/libpf_kernels_ref.so, and adds test-only accessors
// to its private device state (PfState / GlState live in an anonymous
// namespace of that translation unit, so the accessors must be in the same
// translation unit).  Tests use it on the GPU to feed the reference and this
// project's library identical inputs and compare their outputs.  The product
// never links or loads it.
//
// Build: oracle/build.py (PF_REF_SOURCE names the reference's
// src/cuda/pf_kernels.cu).
#ifndef PF_REF_SOURCE
#error "PF_REF_SOURCE must name the reference src/cuda/pf_kernels.cu"
#endif
#include PF_REF_SOURCE

extern "C" {

// Overwrite positions (3n, xyz) / quaternions (4n, w first) / weights (n).
int ref_set_state(void* h, const float* pos3n, const float* quat4n,
                  const float* w) {
    auto* s = static_cast<PfState*>(h);
    if (!s || s->n <= 0) return -1;
    const size_t n = (size_t)s->n;
    if (cudaMemcpy(s->d_pos, pos3n, 3 * sizeof(float) * n,
                   cudaMemcpyHostToDevice) != cudaSuccess)
        return -1;
    if (cudaMemcpy(s->d_att, quat4n, 4 * sizeof(float) * n,
                   cudaMemcpyHostToDevice) != cudaSuccess)
        return -1;
    if (w && cudaMemcpy(s->d_w, w, sizeof(float) * n, cudaMemcpyHostToDevice) !=
                 cudaSuccess)
        return -1;
    return 0;
}

int ref_get_w(void* h, float* w) {
    auto* s = static_cast<PfState*>(h);
    if (!s || s->n <= 0) return -1;
    return cudaMemcpy(w, s->d_w, sizeof(float) * s->n, cudaMemcpyDeviceToHost) ==
                   cudaSuccess
               ? 0
               : -1;
}

int ref_get_ll(void* h, float* ll) {
    auto* s = static_cast<PfState*>(h);
    if (!s || s->n <= 0) return -1;
    return cudaMemcpy(ll, s->d_ll, sizeof(float) * s->n,
                      cudaMemcpyDeviceToHost) == cudaSuccess
               ? 0
               : -1;
}

int ref_get_cum(void* h, double* cum) {
    auto* s = static_cast<PfState*>(h);
    if (!s || s->n <= 0) return -1;
    return cudaMemcpy(cum, s->d_cum, sizeof(double) * s->n,
                      cudaMemcpyDeviceToHost) == cudaSuccess
               ? 0
               : -1;
}

unsigned long long ref_get_lcg(void* h) {
    auto* s = static_cast<PfState*>(h);
    return s ? s->lcg : 0ull;
}

int ref_set_lcg(void* h, unsigned long long lcg) {
    auto* s = static_cast<PfState*>(h);
    if (!s) return -1;
    s->lcg = lcg;
    return 0;
}

unsigned long long ref_get_gen(void* h) {
    auto* s = static_cast<PfState*>(h);
    return s ? (unsigned long long)s->gen : 0ull;
}

int ref_gl_set_hyps(void* h, const float* hyp3n, int n) {
    auto* g = static_cast<GlState*>(h);
    if (!g || n <= 0 || n > g->cap_hyp) return -1;
    g->nh = n;
    if (cudaMemcpy(g->d_hyp, hyp3n, 3 * sizeof(float) * (size_t)n,
                   cudaMemcpyHostToDevice) != cudaSuccess)
        return -1;
    k_gl_iota<<<(n + 255) / 256, 256>>>(g->d_vals, n);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

int ref_gl_get_hyps(void* h, float* hyp3n) {
    auto* g = static_cast<GlState*>(h);
    if (!g || g->nh <= 0) return -1;
    return cudaMemcpy(hyp3n, g->d_hyp, 3 * sizeof(float) * (size_t)g->nh,
                      cudaMemcpyDeviceToHost) == cudaSuccess
               ? 0
               : -1;
}

int ref_gl_get_caer(void* h, float* caer) {
    auto* g = static_cast<GlState*>(h);
    if (!g || g->nh <= 0) return -1;
    return cudaMemcpy(caer, g->d_caer, sizeof(float) * (size_t)g->nh,
                      cudaMemcpyDeviceToHost) == cudaSuccess
               ? 0
               : -1;
}

int ref_gl_set_caer(void* h, const float* caer, int n) {
    auto* g = static_cast<GlState*>(h);
    if (!g || n <= 0 || n > g->cap_hyp) return -1;
    g->nh = n;
    if (cudaMemcpy(g->d_caer, caer, sizeof(float) * (size_t)n,
                   cudaMemcpyHostToDevice) != cudaSuccess)
        return -1;
    k_gl_iota<<<(n + 255) / 256, 256>>>(g->d_vals, n);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

// Sorted hypothesis indices left by the last pfgl_topk (first n).
int ref_gl_get_sorted(void* h, int* vals, int n) {
    auto* g = static_cast<GlState*>(h);
    if (!g || n <= 0 || n > g->nh) return -1;
    return cudaMemcpy(vals, g->d_vals2, sizeof(int) * (size_t)n,
                      cudaMemcpyDeviceToHost) == cudaSuccess
               ? 0
               : -1;
}

}  // extern "C"
