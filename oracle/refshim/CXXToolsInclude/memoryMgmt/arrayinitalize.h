/* Test infrastructure (oracle build only): stand-in for CXX_TOOLS_LIB's
 * arrayInitialize (used e.g. at CBM_STATE_LIB_DEV/src/state/innetconnectivitystate.cpp:650). */
#ifndef CBM_REFSHIM_ARRAYINIT_H
#define CBM_REFSHIM_ARRAYINIT_H
template<typename T> void arrayInitialize(T *arr, T val, unsigned long long n)
{
	for (unsigned long long i = 0; i < n; i++) arr[i] = val;
}
#endif
