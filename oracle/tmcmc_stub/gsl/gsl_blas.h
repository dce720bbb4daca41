#include "../gsl_stub.h"
