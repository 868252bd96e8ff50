/* Forwards to the serial PETSc shim (test infrastructure only). */
#include "petscshim.h"
