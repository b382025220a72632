/* Compile-only stand-in for <mpi.h>, for building the reference's SOA header
 * (gSoFa_SOAComparison/symbfact_warp_centric_new_scheduling.cuh) into the
 * single-rank supernode harness oracle/ref_soa_supernodes.cu.  TEST
 * INFRASTRUCTURE ONLY.  The harness never calls the header's MPI code paths
 * (its work stealing, compiled in but unused); these declarations only let
 * them compile, and every function is a no-op for one rank. */
#ifndef GSOFA_REF_MPI_STUB_H
#define GSOFA_REF_MPI_STUB_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef int MPI_Win;
typedef int MPI_Info;
typedef int MPI_Op;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_CHAR 3
#define MPI_REQUEST_NULL 0
#define MPI_INFO_NULL 0
#define MPI_ANY_SOURCE (-1)
#define MPI_LOCK_EXCLUSIVE 1
#define MPI_SUM 0
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { return 0; }
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { return 0; }
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return 0; }
static inline int MPI_Test(MPI_Request*, int* flag, MPI_Status*) { *flag = 1; return 0; }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Type_create_struct(int, const int*, const MPI_Aint*, const MPI_Datatype*, MPI_Datatype*) { return 0; }
static inline int MPI_Type_commit(MPI_Datatype*) { return 0; }
static inline int MPI_Win_create(void*, MPI_Aint, int, MPI_Info, MPI_Comm, MPI_Win*) { return 0; }
static inline int MPI_Win_lock(int, int, int, MPI_Win) { return 0; }
static inline int MPI_Win_unlock(int, MPI_Win) { return 0; }
static inline int MPI_Win_flush_local(int, MPI_Win) { return 0; }
static inline int MPI_Win_flush_all(MPI_Win) { return 0; }
static inline int MPI_Fetch_and_op(const void*, void*, MPI_Datatype, int, MPI_Aint, MPI_Op, MPI_Win) { return 0; }
#endif
