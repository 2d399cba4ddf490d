// graptor/target/vt_longint.h for sources written against Graptor: vector
// traits of the reference's multi-word integers, not used on the device path;
// the include is kept valid.
#ifndef GRAPTOR_B200_COMPAT_VT_LONGINT_H
#define GRAPTOR_B200_COMPAT_VT_LONGINT_H
#include "graptor/graptor.h"
#endif
