/* Test infrastructure (oracle build only): stand-in for CXX_TOOLS_LIB's
 * dynamic 2-D array helpers.  The reference relies on the rows being one
 * contiguous block (its stateRW calls read and write arr[0] for rows*cols
 * elements, e.g. CBM_STATE_LIB_DEV/src/state/innetconnectivitystate.cpp:540),
 * so the storage is a single allocation plus a row-pointer table. */
#ifndef CBM_REFSHIM_DYNAMIC2DARRAY_H
#define CBM_REFSHIM_DYNAMIC2DARRAY_H
#include <cstddef>

template<typename T> T **allocate2DArray(unsigned long long rows, unsigned long long cols)
{
	T **rowPtr = new T*[rows > 0 ? rows : 1];
	T *block = new T[(rows * cols) > 0 ? rows * cols : 1];
	for (unsigned long long r = 0; r < rows; r++) rowPtr[r] = block + r * cols;
	if (rows == 0) rowPtr[0] = block;
	return rowPtr;
}

template<typename T> void delete2DArray(T **arr)
{
	if (arr == NULL) return;
	delete[] arr[0];
	delete[] arr;
}
#endif
