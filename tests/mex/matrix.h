/* See mex.h (test stand-in). */
#include "mex.h"
