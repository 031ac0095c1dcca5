/* Single-rank MPI runtime: the subset of MPI-3 that the reference driver
 * (mpi/main.cc and the headers it includes, external/indexed_bfs) calls,
 * implemented for a world of exactly one process.  A program linked against
 * it behaves as under `mpiexec -n 1`: collectives copy the caller's own
 * contribution, point-to-point messages go to a self mailbox with tag
 * matching, files are POSIX files.
 *
 * Test and baseline infrastructure: it exists so that the reference's own
 * CPU BFS can be built here unchanged (oracle/ref/make_reference.sh) and
 * serve as the oracle and the timed CPU baseline.  Nothing in the B200
 * engine links it. */
#ifndef ORACLE_REF_SHIM_MPI_H
#define ORACLE_REF_SHIM_MPI_H

/* A real mpi.h pulls these in; the reference relies on it. */
#include <pthread.h>
#include <stddef.h>
#include <stdint.h>
#include <time.h>
#ifdef __cplusplus
#include <stdexcept>
#endif

#define MPI_VERSION 3
#define MPI_SUBVERSION 1

typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_File;
typedef int MPI_Request;
typedef int MPI_Errhandler;
typedef long MPI_Aint;
typedef long long MPI_Offset;
typedef long long MPI_Count;

typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  long long shim_bytes; /* bytes delivered, for MPI_Get_count */
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_UNDEFINED (-32766)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_PROC_NULL (-2)
#define MPI_ROOT (-3)
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_MAX_ERROR_STRING 256

#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)
#define MPI_BOTTOM ((void*)0)

#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3

/* Handles.  0 is the null handle of every kind. */
#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_REQUEST_NULL 0
#define MPI_INFO_NULL 0
#define MPI_FILE_NULL 0
#define MPI_ERRORS_ARE_FATAL 1
#define MPI_ERRORS_RETURN 2
#define MPI_OP_NULL 0

/* Predefined datatypes (ids below MPI_SHIM_FIRST_USER_TYPE). */
#define MPI_DATATYPE_NULL 0
#define MPI_CHAR 1
#define MPI_SIGNED_CHAR 2
#define MPI_UNSIGNED_CHAR 3
#define MPI_BYTE 4
#define MPI_SHORT 5
#define MPI_UNSIGNED_SHORT 6
#define MPI_INT 7
#define MPI_UNSIGNED 8
#define MPI_LONG 9
#define MPI_UNSIGNED_LONG 10
#define MPI_LONG_LONG 11
#define MPI_LONG_LONG_INT 11
#define MPI_UNSIGNED_LONG_LONG 12
#define MPI_FLOAT 13
#define MPI_DOUBLE 14
#define MPI_LONG_DOUBLE 15
#define MPI_LONG_INT 16
#define MPI_DOUBLE_INT 17
#define MPI_2INT 18
#define MPI_C_BOOL 19
#define MPI_CXX_BOOL 20
#define MPI_INT8_T 21
#define MPI_INT16_T 22
#define MPI_INT32_T 23
#define MPI_INT64_T 24
#define MPI_UINT8_T 25
#define MPI_UINT16_T 26
#define MPI_UINT32_T 27
#define MPI_UINT64_T 28
#define MPI_AINT 29
#define MPI_OFFSET 30
#define MPI_COUNT 31
#define MPI_FLOAT_INT 32
#define MPI_SHIM_FIRST_USER_TYPE 64

/* Reduction operations: with one rank every reduction is the identity on
 * the caller's data, so the operation is only checked for validity. */
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_SUM 3
#define MPI_PROD 4
#define MPI_LAND 5
#define MPI_BAND 6
#define MPI_LOR 7
#define MPI_BOR 8
#define MPI_LXOR 9
#define MPI_BXOR 10
#define MPI_MAXLOC 11
#define MPI_MINLOC 12
#define MPI_REPLACE 13

/* File access modes. */
#define MPI_MODE_RDONLY 2
#define MPI_MODE_RDWR 8
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_MODE_EXCL 64
#define MPI_MODE_DELETE_ON_CLOSE 16
#define MPI_MODE_UNIQUE_OPEN 32
#define MPI_MODE_APPEND 128
#define MPI_MODE_SEQUENTIAL 256
/* One-sided assertion flags (declared by the reference's validator). */
#define MPI_MODE_NOCHECK 1024
#define MPI_MODE_NOSTORE 2048
#define MPI_MODE_NOPUT 4096
#define MPI_MODE_NOPRECEDE 8192
#define MPI_MODE_NOSUCCEED 16384

#ifdef __cplusplus
extern "C" {
#endif

/* Environment */
int MPI_Init(int* argc, char*** argv);
int MPI_Init_thread(int* argc, char*** argv, int required, int* provided);
int MPI_Initialized(int* flag);
int MPI_Finalized(int* flag);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int errorcode);
int MPI_Query_thread(int* provided);
int MPI_Is_thread_main(int* flag);
int MPI_Get_processor_name(char* name, int* resultlen);
int MPI_Error_string(int errorcode, char* string, int* resultlen);
double MPI_Wtime(void);
double MPI_Wtick(void);
int MPI_Alloc_mem(MPI_Aint size, MPI_Info info, void* baseptr);
int MPI_Free_mem(void* base);

/* Communicators */
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* newcomm);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* newcomm);
int MPI_Comm_free(MPI_Comm* comm);
int MPI_Comm_set_errhandler(MPI_Comm comm, MPI_Errhandler errhandler);

/* Datatypes */
int MPI_Type_contiguous(int count, MPI_Datatype oldtype, MPI_Datatype* newtype);
int MPI_Type_create_struct(int count, const int blocklengths[], const MPI_Aint displacements[],
                           const MPI_Datatype types[], MPI_Datatype* newtype);
int MPI_Type_create_resized(MPI_Datatype oldtype, MPI_Aint lb, MPI_Aint extent,
                            MPI_Datatype* newtype);
int MPI_Type_commit(MPI_Datatype* datatype);
int MPI_Type_free(MPI_Datatype* datatype);
int MPI_Type_size(MPI_Datatype datatype, int* size);
int MPI_Type_get_extent(MPI_Datatype datatype, MPI_Aint* lb, MPI_Aint* extent);
int MPI_Get_count(const MPI_Status* status, MPI_Datatype datatype, int* count);

/* Point to point (self mailbox) */
int MPI_Send(const void* buf, int count, MPI_Datatype datatype, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void* buf, int count, MPI_Datatype datatype, int source, int tag, MPI_Comm comm,
             MPI_Status* status);
int MPI_Isend(const void* buf, int count, MPI_Datatype datatype, int dest, int tag, MPI_Comm comm,
              MPI_Request* request);
int MPI_Irecv(void* buf, int count, MPI_Datatype datatype, int source, int tag, MPI_Comm comm,
              MPI_Request* request);
int MPI_Sendrecv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void* recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status* status);
int MPI_Send_init(const void* buf, int count, MPI_Datatype datatype, int dest, int tag,
                  MPI_Comm comm, MPI_Request* request);
int MPI_Recv_init(void* buf, int count, MPI_Datatype datatype, int source, int tag, MPI_Comm comm,
                  MPI_Request* request);
int MPI_Start(MPI_Request* request);
int MPI_Startall(int count, MPI_Request requests[]);
int MPI_Request_free(MPI_Request* request);
int MPI_Test(MPI_Request* request, int* flag, MPI_Status* status);
int MPI_Testany(int count, MPI_Request requests[], int* index, int* flag, MPI_Status* status);
int MPI_Testall(int count, MPI_Request requests[], int* flag, MPI_Status statuses[]);
int MPI_Testsome(int incount, MPI_Request requests[], int* outcount, int indices[],
                 MPI_Status statuses[]);
int MPI_Wait(MPI_Request* request, MPI_Status* status);
int MPI_Waitany(int count, MPI_Request requests[], int* index, MPI_Status* status);
int MPI_Waitall(int count, MPI_Request requests[], MPI_Status statuses[]);
int MPI_Iprobe(int source, int tag, MPI_Comm comm, int* flag, MPI_Status* status);

/* Collectives */
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void* buffer, int count, MPI_Datatype datatype, int root, MPI_Comm comm);
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype, MPI_Op op,
               int root, MPI_Comm comm);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype, MPI_Op op,
                  MPI_Comm comm);
int MPI_Reduce_scatter(const void* sendbuf, void* recvbuf, const int recvcounts[],
                       MPI_Datatype datatype, MPI_Op op, MPI_Comm comm);
int MPI_Reduce_scatter_block(const void* sendbuf, void* recvbuf, int recvcount,
                             MPI_Datatype datatype, MPI_Op op, MPI_Comm comm);
int MPI_Scan(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype, MPI_Op op,
             MPI_Comm comm);
int MPI_Exscan(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype, MPI_Op op,
               MPI_Comm comm);
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
               int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Gatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                const int recvcounts[], const int displs[], MPI_Datatype recvtype, int root,
                MPI_Comm comm);
int MPI_Scatter(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Scatterv(const void* sendbuf, const int sendcounts[], const int displs[],
                 MPI_Datatype sendtype, void* recvbuf, int recvcount, MPI_Datatype recvtype,
                 int root, MPI_Comm comm);
int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                  int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Allgatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                   const int recvcounts[], const int displs[], MPI_Datatype recvtype,
                   MPI_Comm comm);
int MPI_Alltoall(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                 int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Alltoallv(const void* sendbuf, const int sendcounts[], const int sdispls[],
                  MPI_Datatype sendtype, void* recvbuf, const int recvcounts[],
                  const int rdispls[], MPI_Datatype recvtype, MPI_Comm comm);

/* Files (POSIX) */
int MPI_File_open(MPI_Comm comm, const char* filename, int amode, MPI_Info info, MPI_File* fh);
int MPI_File_close(MPI_File* fh);
int MPI_File_delete(const char* filename, MPI_Info info);
int MPI_File_set_atomicity(MPI_File fh, int flag);
int MPI_File_set_errhandler(MPI_File file, MPI_Errhandler errhandler);
int MPI_File_set_size(MPI_File fh, MPI_Offset size);
int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype filetype,
                      const char* datarep, MPI_Info info);
int MPI_File_read_at(MPI_File fh, MPI_Offset offset, void* buf, int count, MPI_Datatype datatype,
                     MPI_Status* status);
int MPI_File_write_at(MPI_File fh, MPI_Offset offset, const void* buf, int count,
                      MPI_Datatype datatype, MPI_Status* status);
int MPI_File_iread_at(MPI_File fh, MPI_Offset offset, void* buf, int count, MPI_Datatype datatype,
                      MPI_Request* request);
int MPI_File_iwrite_at(MPI_File fh, MPI_Offset offset, const void* buf, int count,
                       MPI_Datatype datatype, MPI_Request* request);

#ifdef __cplusplus
}
#endif

#endif /* ORACLE_REF_SHIM_MPI_H */
