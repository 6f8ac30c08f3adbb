// Production FX32 Mobile V2 substep kernels (FAST = true instantiations):
// the single-grid strip kernel, its persistent substep loop and the
// batched-patch kernel.
//
// This translation unit is compiled WITH FMA contraction (nvcc's default
// -fmad=true), unlike soilb200.cu, whose FP64 parity kernels and FX32 mirror
// kernels must keep every multiply and add separately rounded.  The kernel
// body is the register-streaming strip stencil of sb_fv.cuh; FAST selects the
// approximate reciprocal and square root.  Heights stay integer quanta and
// every face mass flux is an integer applied with opposite signs to its two
// cells, so mass is still exact; the float rounding differences against the
// mirror stay far inside the FX32 bound against FP64 (1e-5 m).
//
// soilb200.cu never names fv_stream_kernel<true>, fv_loop_kernel<true> or
// batch_fv_kernel<true> (it would instantiate them under -fmad=false there);
// it takes their addresses from here.
#include "sb_batch_fv.cuh"
#include "sb_fv.cuh"

namespace sb {

const void* fv_stream_fast_kernel() { return reinterpret_cast<const void*>(&fv_stream_kernel<true>); }
const void* batch_fv_fast_kernel() { return reinterpret_cast<const void*>(&batch_fv_kernel<true>); }
const void* fv_loop_fast_kernel() { return reinterpret_cast<const void*>(&fv_loop_kernel<true>); }

}  // namespace sb
