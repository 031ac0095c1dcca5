/* Declaration-only single-rank MPI header: just enough names for the
 * reference's generator header (generator/graph_generator.hpp) to compile
 * so that its edge generator and make_random_numbers can produce golden
 * vectors.  Nothing here is called by the golden-vector driver. */
#ifndef ORACLE_REF_STUB_MPI_H
#define ORACLE_REF_STUB_MPI_H
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <time.h>
#include <string.h>
#include <stdlib.h>
#include <inttypes.h>
#include <unistd.h>
#include <omp.h>
#ifdef __cplusplus
#include <stdexcept>
#endif
#define IMD_OUT stderr
#define MPI_VERSION 3
#define MPI_SUBVERSION 1
typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_File;
typedef int MPI_Request;
typedef long long MPI_Offset;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_DATATYPE_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_INFO_NULL 0
#define MPI_MODE_RDWR 1
#define MPI_MODE_CREATE 2
#define MPI_MODE_DELETE_ON_CLOSE 4
#define MPI_MODE_UNIQUE_OPEN 8
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_INT64_T 11
#define MPI_UINT64_T 12
#define MPI_UINT32_T 13
#define MPI_UINT16_T 14
#define MPI_AINT 15
#define MPI_MAX 1
#define MPI_INT 16
#define MPI_BYTE 17
#ifdef __cplusplus
extern "C" {
#endif
int MPI_Type_contiguous(int, MPI_Datatype, MPI_Datatype*);
int MPI_Type_commit(MPI_Datatype*);
int MPI_Type_free(MPI_Datatype*);
int MPI_Type_create_struct(int, const int*, const MPI_Aint*, const MPI_Datatype*, MPI_Datatype*);
int MPI_Allreduce(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm);
int MPI_Wait(MPI_Request*, MPI_Status*);
int MPI_File_open(MPI_Comm, char*, int, MPI_Info, MPI_File*);
int MPI_File_close(MPI_File*);
int MPI_File_set_atomicity(MPI_File, int);
int MPI_File_set_view(MPI_File, MPI_Offset, MPI_Datatype, MPI_Datatype, char*, MPI_Info);
int MPI_File_iread_at(MPI_File, MPI_Offset, void*, int, MPI_Datatype, MPI_Request*);
int MPI_File_read_at(MPI_File, MPI_Offset, void*, int, MPI_Datatype, MPI_Status*);
int MPI_File_write_at(MPI_File, MPI_Offset, const void*, int, MPI_Datatype, MPI_Status*);
#ifdef __cplusplus
}
template <typename T> struct MpiTypeOf;
struct StubMpiGlobals {
  int rank_2d = 0, size_2d = 1;
  bool isMaster() const { return true; }
};
extern StubMpiGlobals mpi;
void print_with_prefix(const char* fmt, ...);
void* cache_aligned_xmalloc(size_t size);
#endif
#endif
