// graptor/api.h for sources written against Graptor (see graptor/graptor.h).
#include "graptor/graptor.h"
