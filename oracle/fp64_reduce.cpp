// fp64_reduce.cpp -- TEST INFRASTRUCTURE ONLY (oracle).
//
// Replacement for the reference's Clarity_ReduceSum
// (src/ComputePrimitives.cxx:44-82) used only in liboracle_ref_fp64sum.so:
// the same serial loop over the buffer, but accumulated in double and
// rounded to float once.  The reference's serial float accumulator loses
// about 1e-3 relative accuracy over 33.5M voxels; this variant isolates
// that one difference so the rest of the reference algorithm can be compared
// at 1e-5.
#include "Clarity.h"
#include "ComputePrimitives.h"  // declares it with C++ linkage

ClarityResult_t Clarity_ReduceSum(float* result, float* buffer, int n) {
  double sum = 0.0;
  for (int i = 0; i < n; i++) sum += buffer[i];
  *result = (float)sum;
  return CLARITY_SUCCESS;
}
