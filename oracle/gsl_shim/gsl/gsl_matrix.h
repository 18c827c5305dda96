#include "gsl_eigen.h"
