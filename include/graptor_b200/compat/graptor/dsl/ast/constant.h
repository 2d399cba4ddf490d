// graptor/dsl/ast/constant.h for sources written against Graptor: the
// expression constants (_0, _1, _1s, _c) live in graptor_b200/api.h.
#ifndef GRAPTOR_B200_COMPAT_DSL_AST_CONSTANT_H
#define GRAPTOR_B200_COMPAT_DSL_AST_CONSTANT_H
#include "graptor/graptor.h"
#endif
