#include "gsl_vector.h"
