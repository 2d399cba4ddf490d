// graptor/longint.h for sources written against Graptor: the multi-word
// integer type of the reference's SIMD layer is not used on the device path
// (bit strings are one uint32 word per vertex); the include is kept valid.
#ifndef GRAPTOR_B200_COMPAT_LONGINT_H
#define GRAPTOR_B200_COMPAT_LONGINT_H
#include "graptor/graptor.h"
#endif
