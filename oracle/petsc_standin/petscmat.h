/* Stand-in for PETSc's petscmat.h when compiling the reference's PETSc-free
 * element sources (LocalAssembly*.hpp only use PetscScalar from it).
 * Test infrastructure only. */
#ifndef IGA_ORACLE_PETSCMAT_STANDIN_H
#define IGA_ORACLE_PETSCMAT_STANDIN_H
typedef double PetscScalar;
typedef int PetscInt;
#endif
