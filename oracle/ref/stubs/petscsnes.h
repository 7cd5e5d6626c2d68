/* petscsnes.h -- stand-in for the PETSc 2.3.3 header that the reference's
 * comobject_mpi.hpp includes, for building the reference's own kernel and
 * operator sources at one rank (test infrastructure: oracle/_ref only).
 *
 * Those sources use nothing of PETSc but an MPI communicator handle, rank and
 * size queries (always rank 0 of 1 here) and the CHKERRQ / SETERRQ error
 * macros, which return the error code from the calling function as PETSc's
 * do. */
#ifndef FMMG_REF_STUB_PETSCSNES_H_
#define FMMG_REF_STUB_PETSCSNES_H_

typedef int MPI_Comm;
static const MPI_Comm PETSC_COMM_WORLD = 0;
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }

#define CHKERRQ(e) do { if (e) return (e); } while (0)
#define SETERRQ(n, s) return (n)

#endif
