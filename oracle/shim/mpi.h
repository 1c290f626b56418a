/*
 * Single-rank MPI shim for building the reference HOS hot-path sources on a
 * host without MPI.  TEST INFRASTRUCTURE ONLY: this header exists so that
 * Csource/2dpar/{hosm_2d_par,operators_par,time_schemes_par,fft_routines_2d_par}.c
 * compile unchanged into the CPU oracle.  Nothing in the product links it.
 *
 * Only what those translation units and euler_2d_par.h:62-66 name is declared:
 * the communicator/info types, MPI_Reduce (time_schemes_par.c:76) and the
 * constants it is called with.
 */
#ifndef HOS_ORACLE_SHIM_MPI_H
#define HOS_ORACLE_SHIM_MPI_H

typedef int MPI_Comm;
typedef int MPI_Info;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_FLOAT 1
#define MPI_DOUBLE 2
#define MPI_SUM 1

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Barrier(MPI_Comm comm);
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type,
               MPI_Op op, int root, MPI_Comm comm);

#endif
