// Shim around the reference's own implicit cooling solver
// (11_Dec_2022/GPU_sph/With_cooling/Model_C/myPhotoLibsGPU.h:588-686),
// compiled as host C++ straight from the reference tree into oracle/_ref/.
// It exports DoCooling and coolingRateFromU with C linkage so the tests can
// pin the FP32 bisection restatement in sph_oracle.c against the reference.
// Test infrastructure only.
#define __host__
#define __device__
#include "myPhotoLibsGPU.h"

extern "C" float ref_DoCooling(float rho, float u_old, float dt, float XH)
{
    return DoCooling(rho, u_old, dt, XH);
}

extern "C" float ref_coolingRateFromU(float u, float nH, float XH)
{
    return coolingRateFromU(u, nH, XH);
}
