/* Test infrastructure (oracle build only): stand-in for CXX_TOOLS_LIB's
 * arrayCopy (used e.g. at CBM_STATE_LIB_DEV/src/state/innetconnectivitystate.cpp:62). */
#ifndef CBM_REFSHIM_ARRAYCOPY_H
#define CBM_REFSHIM_ARRAYCOPY_H
template<typename T> void arrayCopy(T *dst, const T *src, unsigned long long n)
{
	for (unsigned long long i = 0; i < n; i++) dst[i] = src[i];
}
#endif
