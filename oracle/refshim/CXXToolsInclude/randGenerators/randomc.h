/* Test infrastructure (oracle build only): the reference includes randomc.h
 * for the generator declarations; they live in sfmt.h here. */
#include "sfmt.h"
