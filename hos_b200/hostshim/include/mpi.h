/*
 * mpi.h -- single-rank MPI for the reference's host driver on one GPU.
 *
 * The reference's driver (Csource/2dpar/main_2d_par.c) and HDF5 routines
 * (hdf5_routines_2d_par.c) are MPI programs.  On one GPU every field lives
 * in one process, so a host without an MPI installation can build them
 * against this header and libhos_hostshim.so: the world has one rank (0),
 * barriers return at once and reductions copy.  Only what those files and
 * the headers they include name is declared (main_2d_par.c:69-77,107,373;
 * euler_2d_par.h:62-66; time_schemes_par.c:76).  A host that has MPI uses its
 * own mpi.h and library instead.
 */
#ifndef HOS_HOSTSHIM_MPI_H
#define HOS_HOSTSHIM_MPI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Info;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_FLOAT 1
#define MPI_DOUBLE 2
#define MPI_INT 3
#define MPI_SUM 1
#define MPI_SUCCESS 0
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3

int MPI_Init(int* argc, char*** argv);
int MPI_Init_thread(int* argc, char*** argv, int required, int* provided);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Barrier(MPI_Comm comm);
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, int root,
               MPI_Comm comm);

#ifdef __cplusplus
}
#endif

#endif
