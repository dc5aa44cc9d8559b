/* Test infrastructure (oracle build only): stand-in for the un-vendored
 * CXX_TOOLS_LIB header that the reference includes as
 * <CXXToolsInclude/stdDefinitions/pstdint.h>
 * (e.g. CBM_CORE_LIB_MGPU_DEV/CBMCoreInclude/interface/cbmsimcore.h:20).
 * Only the fixed-width aliases the reference uses are provided. */
#ifndef CBM_REFSHIM_PSTDINT_H
#define CBM_REFSHIM_PSTDINT_H
#include <stdint.h>
typedef int8_t ct_int8_t;
typedef uint8_t ct_uint8_t;
typedef int16_t ct_int16_t;
typedef uint16_t ct_uint16_t;
typedef int32_t ct_int32_t;
typedef uint32_t ct_uint32_t;
typedef int64_t ct_int64_t;
typedef uint64_t ct_uint64_t;
#endif
