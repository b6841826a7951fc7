/* Drop-in name for programs written against the reference's libsmoldyn.h
 * (source/Smoldyn/libsmoldyn.h): `#include <libsmoldyn.h>` with this
 * directory on the include path and `-lsmoldyn_b200` at link time builds
 * them against the B200 engine.  Everything is declared in smoldyn_b200.h. */
#ifndef LIBSMOLDYN_B200_COMPAT_H
#define LIBSMOLDYN_B200_COMPAT_H
#include "smoldyn_b200.h"
#endif
