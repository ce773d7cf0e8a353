/* Forwarding header: see petsc_shim.h (test-oracle shim only). */
#include "petsc_shim.h"
