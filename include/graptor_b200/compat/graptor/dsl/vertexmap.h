// graptor/dsl/vertexmap.h for sources written against Graptor: the lazy
// executor lives in graptor_b200/api.h.
#include "graptor/graptor.h"
