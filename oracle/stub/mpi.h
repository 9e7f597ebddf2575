/* Minimal MPI type stub so that the reference's single-rank CPU sources
 * (w-stacking.cu, phase_correction.cu compiled as C) build without an MPI
 * installation.  Only the type names those headers mention are provided; no
 * MPI function is called on the CPU wstack / phase_correction path.
 *
 * Test infrastructure only: used by oracle/Makefile to build oracle/_ref.
 */
#ifndef RICK_ORACLE_MPI_STUB_H
#define RICK_ORACLE_MPI_STUB_H
typedef int  MPI_Comm;
typedef int  MPI_Win;
typedef long MPI_Aint;
typedef int  MPI_Request;
typedef int  MPI_Datatype;
typedef int  MPI_Info;
typedef int  MPI_Op;
/* gridding.c's NORMALIZE_UVW block reduces its extrema over the ranks; with one
 * rank and MPI_IN_PLACE that reduction leaves the buffers as they are
 * (stub/ref_norm_stubs.c). */
#define MPI_IN_PLACE   ((void *)1)
#define MPI_DOUBLE     ((MPI_Datatype)0)
#define MPI_MIN        ((MPI_Op)0)
#define MPI_MAX        ((MPI_Op)1)
#define MPI_COMM_WORLD ((MPI_Comm)0)
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype datatype, MPI_Op op,
                  MPI_Comm comm);
#endif
