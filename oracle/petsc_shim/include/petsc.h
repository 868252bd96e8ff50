/* Umbrella PETSc header of the serial shim (test infrastructure only). */
#pragma once
#include "petscshim.h"
