// ocfd_sweep4_f32.cu -- FP32 instances of the in-line walk (precision form)
// and the FP32 fix-up of the cells the FP32 UP7 walk defers.
#include "ocfd_sweep4.cuh"

namespace ocfd {

using namespace walk4;

cudaError_t sweep4_dir_f32(const Params &p, int dir, cudaStream_t st) { return dir4r<float>(p, dir, st); }

// fix-up of the cells the FP32 call-free UP7 walk deferred in direction dir
cudaError_t launch_sweep4_fix(const Params &p, int dir, cudaStream_t st) {
    if (!(p.scheme_invis == 310 && p.charteric)) return cudaErrorNotSupported;
    const bool u = p.uniform_metrics, e0 = p.epsl_sw == 0.0;
#define OCFD_FIX4(D, U, E) k_sweep4_fix<D, U, E, float><<<2 * 148, 32 * FIX4W, 0, st>>>(p)
    if (dir == 0)      { if (u && e0) OCFD_FIX4(0, true, true); else if (u) OCFD_FIX4(0, true, false); else OCFD_FIX4(0, false, false); }
    else if (dir == 1) { if (u && e0) OCFD_FIX4(1, true, true); else if (u) OCFD_FIX4(1, true, false); else OCFD_FIX4(1, false, false); }
    else               { if (u && e0) OCFD_FIX4(2, true, true); else if (u) OCFD_FIX4(2, true, false); else OCFD_FIX4(2, false, false); }
#undef OCFD_FIX4
    return cudaGetLastError();
}

}  // namespace ocfd
