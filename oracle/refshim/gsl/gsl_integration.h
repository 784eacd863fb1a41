/* see gsl_shim.h */
#include "gsl_shim.h"
