/* Test infrastructure (oracle build only): stand-in for CXX_TOOLS_LIB's
 * float-array validation (CBM_STATE_LIB_DEV/src/state/innetactivitystate.cpp:163-182):
 * true when every element is finite. */
#ifndef CBM_REFSHIM_ARRAYVALIDATE_H
#define CBM_REFSHIM_ARRAYVALIDATE_H
#include <cmath>
inline bool validateFloatArray(const float *arr, unsigned long long n)
{
	for (unsigned long long i = 0; i < n; i++) if (!std::isfinite(arr[i])) return false;
	return true;
}
inline bool validate2DfloatArray(float **arr, unsigned long long n)
{
	return validateFloatArray(arr[0], n);
}
#endif
