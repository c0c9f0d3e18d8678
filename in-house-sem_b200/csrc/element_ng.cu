// Element-forces launchers for one number of GLL points, selected at compile
// time with -DINSEM_NG=<2..9>; the build compiles this file once per value.
#include "element_kernels.cuh"

#ifndef INSEM_NG
#error "compile with -DINSEM_NG=<number of GLL points>"
#endif

#define INSEM_CAT2(a, b) a##b
#define INSEM_CAT(a, b) INSEM_CAT2(a, b)

namespace insem_b200 {

void INSEM_CAT(launch_element_ng, INSEM_NG)(const ElementLaunch& a) { launch_element_ng<INSEM_NG>(a); }

}  // namespace insem_b200
