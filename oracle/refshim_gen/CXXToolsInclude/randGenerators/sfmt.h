/* Test infrastructure (oracle "gen" build only): forwards to the SFMT copy the
 * reference vendors (CBM_Cart_On_Cart/includes/sfmt.h), which the recipe in
 * oracle/Makefile compiles in place, so that reference connectivity
 * generation reproduces the reference's own random sequence. */
#include CBM_REF_SFMT_HEADER
