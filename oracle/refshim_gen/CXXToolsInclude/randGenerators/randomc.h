/* Test infrastructure (oracle "gen" build only): see sfmt.h beside this file. */
#include CBM_REF_SFMT_HEADER
