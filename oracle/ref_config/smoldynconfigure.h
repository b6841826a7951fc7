/* Build settings for compiling the reference Smoldyn sources as the test
 * oracle (Linux, no OpenGL, no TIFF, no NextSubvolume, no VTK, no VCell).
 * Only macros are defined here; no reference code is carried. */
#ifndef SMOLDYN_ORACLE_CONFIGURE_H
#define SMOLDYN_ORACLE_CONFIGURE_H
#define NIX_BUILD 1
#define HAVE_MEMORY_H 1
#define VERSION "2.76.dev-oracle"
#define BNG2_PATH "BNG2.pl"
#endif
