// ocfd_sweep4.cu -- the in-line walk's entry points and its FP64 instances
// (the kernels are in ocfd_sweep4.cuh; FP32 instances in ocfd_sweep4_f32.cu).
#include "ocfd_sweep4.cuh"

namespace ocfd {

cudaError_t sweep4_dir_f32(const Params &p, int dir, cudaStream_t st);


// the schemes this walk covers: the hybrid scheme with characteristic
// projection, WENO7 on the flux components
bool sweeps4_supported(const Params &p) {
    return (p.scheme_invis == 310 && p.charteric) || (p.scheme_invis == 303 && !p.charteric);
}

// one direction of the walk (one kernel); FP32 in the precision form
cudaError_t launch_sweep4_dir(const Params &p, int dir, cudaStream_t st) {
    if (!sweeps4_supported(p)) return cudaErrorNotSupported;
    return p.mixed ? sweep4_dir_f32(p, dir, st) : walk4::dir4r<double>(p, dir, st);
}

cudaError_t launch_sweeps4(const Params &p, cudaStream_t st) {
    cudaError_t e;
    for (int d = 0; d < 3; d++)
        if ((e = launch_sweep4_dir(p, d, st)) != cudaSuccess) return e;
    return cudaSuccess;
}

}  // namespace ocfd
