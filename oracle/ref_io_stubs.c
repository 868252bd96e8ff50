/*
 * Link stubs for the reference's main.c in oracle/_ref/libchimera_ref_io.so
 * (TEST INFRASTRUCTURE ONLY).  main.c is compiled unmodified (its main()
 * renamed by the preprocessor) for Q_P_Binary_Output, Q_P_Binary_Input and
 * RestartApplication; the functions below are referenced only by its main(),
 * its FSI branch of RestartApplication and its VTK reader, none of which the
 * checkpoint tests run.  Each returns an error if it is ever called.
 */
#include "variables.h"

PetscErrorCode PetscInitialize(int *argc, char ***argv, const char *file, const char *help) {
  (void)argc; (void)argv; (void)file; (void)help;
  return 1;
}
PetscErrorCode PetscFinalize(void) { return 1; }
PetscErrorCode DMDAGetAO() { return 1; }
PetscErrorCode AOApplicationToPetsc() { return 1; }
PetscErrorCode MG_Initial() { return 1; }
PetscErrorCode MG_Finalize() { return 1; }
PetscErrorCode FsiInitialize() { return 1; }
PetscErrorCode FSI_DATA_Input() { return 1; }
PetscErrorCode fish_init() { return 1; }
PetscErrorCode ibm_read_Ansys() { return 1; }
PetscErrorCode ibm_read_ucd() { return 1; }
