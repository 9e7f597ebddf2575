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
#endif
