// raster_ref_nofma.cu -- raster_ref.cu compiled with --use_fast_math and
// -fmad=false (CR_RENDER_REF_MATH_NO_FMA frames): the reference's recipe with
// contraction turned off, which its NVRTC build accepts as --fmad=false after
// --use_fast_math.  Without contracted products the approximate divisions
// and square roots are the only departures from IEEE arithmetic, and both
// builds form them from the same operations, so the visbuffer is the
// reference's bit for bit.
#define CR_REF_RASTER_ENTRY cr_launch_ref_raster_nofma
#include "raster_ref.cu"
