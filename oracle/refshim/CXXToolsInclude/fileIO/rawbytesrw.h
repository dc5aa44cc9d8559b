/* Test infrastructure (oracle build only): stand-in for CXX_TOOLS_LIB's
 * rawBytesRW, which the reference's stateRW functions use to read or write a
 * raw byte block at the stream position
 * (e.g. CBM_STATE_LIB_DEV/src/state/innetactivitystate.cpp:235). */
#ifndef CBM_REFSHIM_RAWBYTESRW_H
#define CBM_REFSHIM_RAWBYTESRW_H
#include <fstream>
inline void rawBytesRW(char *arr, unsigned long long byteLen, bool read, std::fstream &file)
{
	if (read) file.read(arr, (std::streamsize)byteLen);
	else file.write(arr, (std::streamsize)byteLen);
}
#endif
