// Single-rank MPI runtime (see mpi.h): every communicator holds one process
// (rank 0), so a collective is a copy of the caller's own block, a reduction
// is the identity, and a message is matched against the receives this same
// process posts.  Messages are delivered eagerly: a send whose receive is not
// yet posted is buffered in the mailbox and completes at once, which is one
// of the completion orders MPI allows.  The state is guarded by one mutex
// because the reference calls MPI from its communication thread as well as
// from the main thread.
//
// Test and baseline infrastructure only (builds the reference's CPU BFS
// unchanged); the B200 engine never links it.
#include "mpi.h"

#include <fcntl.h>
#include <sched.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <vector>

namespace {

struct TypeInfo {
  bool live = false;
  long size = 0;    // bytes of data (MPI_Type_size)
  long lb = 0;      // lower bound
  long extent = 0;  // stride between consecutive elements
  long align = 1;   // alignment used to pad struct extents
};

struct Message {  // a buffered send waiting for its receive
  MPI_Comm comm;
  int tag;
  std::vector<char> data;
};

enum ReqKind { kFree = 0, kSend, kRecv, kDone };

struct Request {
  ReqKind kind = kFree;
  bool persistent = false;
  bool active = false;  // persistent requests: started and not completed
  // send or receive arguments
  const void* sbuf = nullptr;
  void* rbuf = nullptr;
  long bytes = 0;  // capacity of the receive buffer / size of the send
  MPI_Comm comm = MPI_COMM_NULL;
  int tag = 0;
  bool complete = false;
  MPI_Status status{};
};

struct FileInfo {
  int fd = -1;
  bool delete_on_close = false;
  std::string path;
  MPI_Offset disp = 0;
  long etype_extent = 1;
};

struct State {
  std::mutex mu;
  std::vector<TypeInfo> types;
  std::vector<Request> reqs;   // index = handle; 0 unused (MPI_REQUEST_NULL)
  std::vector<int> free_reqs;
  std::deque<Message> unexpected;
  std::vector<int> posted_recvs;  // receive requests waiting for a message
  std::vector<bool> comms;        // live communicator handles
  std::vector<FileInfo> files;    // index = handle; 0 unused (MPI_FILE_NULL)
  bool initialized = false, finalized = false;
  State() {
    types.resize(MPI_SHIM_FIRST_USER_TYPE);
    auto basic = [&](int id, long size, long align) {
      types[id].live = true;
      types[id].size = size;
      types[id].extent = size;
      types[id].align = align;
    };
    basic(MPI_CHAR, 1, 1);
    basic(MPI_SIGNED_CHAR, 1, 1);
    basic(MPI_UNSIGNED_CHAR, 1, 1);
    basic(MPI_BYTE, 1, 1);
    basic(MPI_SHORT, sizeof(short), alignof(short));
    basic(MPI_UNSIGNED_SHORT, sizeof(short), alignof(short));
    basic(MPI_INT, sizeof(int), alignof(int));
    basic(MPI_UNSIGNED, sizeof(int), alignof(int));
    basic(MPI_LONG, sizeof(long), alignof(long));
    basic(MPI_UNSIGNED_LONG, sizeof(long), alignof(long));
    basic(MPI_LONG_LONG, sizeof(long long), alignof(long long));
    basic(MPI_UNSIGNED_LONG_LONG, sizeof(long long), alignof(long long));
    basic(MPI_FLOAT, sizeof(float), alignof(float));
    basic(MPI_DOUBLE, sizeof(double), alignof(double));
    basic(MPI_LONG_DOUBLE, sizeof(long double), alignof(long double));
    basic(MPI_C_BOOL, 1, 1);
    basic(MPI_CXX_BOOL, sizeof(bool), alignof(bool));
    basic(MPI_INT8_T, 1, 1);
    basic(MPI_INT16_T, 2, 2);
    basic(MPI_INT32_T, 4, 4);
    basic(MPI_INT64_T, 8, 8);
    basic(MPI_UINT8_T, 1, 1);
    basic(MPI_UINT16_T, 2, 2);
    basic(MPI_UINT32_T, 4, 4);
    basic(MPI_UINT64_T, 8, 8);
    basic(MPI_AINT, sizeof(MPI_Aint), alignof(MPI_Aint));
    basic(MPI_OFFSET, sizeof(MPI_Offset), alignof(MPI_Offset));
    basic(MPI_COUNT, sizeof(MPI_Count), alignof(MPI_Count));
    // pair types of MAXLOC/MINLOC: {value, int} as the C struct lays it out
    struct LI { long a; int b; };
    struct DI { double a; int b; };
    struct FI { float a; int b; };
    struct II { int a; int b; };
    basic(MPI_LONG_INT, sizeof(LI), alignof(LI));
    types[MPI_LONG_INT].size = sizeof(long) + sizeof(int);
    basic(MPI_DOUBLE_INT, sizeof(DI), alignof(DI));
    types[MPI_DOUBLE_INT].size = sizeof(double) + sizeof(int);
    basic(MPI_FLOAT_INT, sizeof(FI), alignof(FI));
    basic(MPI_2INT, sizeof(II), alignof(II));
    reqs.resize(1);
    comms.assign(3, true);
    comms[MPI_COMM_NULL] = false;
    files.resize(1);
  }
};

State& st() {
  static State* s = new State();  // never destroyed: MPI calls may run at exit
  return *s;
}

[[noreturn]] void fatal(const char* what) {
  fprintf(stderr, "[mpi shim] %s\n", what);
  fflush(stderr);
  abort();
}

const TypeInfo& type_of(State& s, MPI_Datatype t) {
  if (t <= 0 || t >= (int)s.types.size() || !s.types[t].live) fatal("invalid datatype");
  return s.types[t];
}

long extent_of(MPI_Datatype t) { return type_of(st(), t).extent; }

void check_comm(State& s, MPI_Comm c) {
  if (c <= 0 || c >= (int)s.comms.size() || !s.comms[c]) fatal("invalid communicator");
}

void check_peer(int rank) {
  if (rank != 0 && rank != MPI_ANY_SOURCE && rank != MPI_PROC_NULL)
    fatal("peer rank out of range in a one-process world");
}

void check_root(int root) {
  if (root != 0) fatal("collective root out of range in a one-process world");
}

// Copies count elements of type t; buffers may overlap (in-place use).
void copy_block(void* dst, const void* src, long count, MPI_Datatype t) {
  if (src == MPI_IN_PLACE || count <= 0 || dst == src) return;
  memmove(dst, src, (size_t)(count * extent_of(t)));
}

int new_request(State& s) {
  int h;
  if (!s.free_reqs.empty()) {
    h = s.free_reqs.back();
    s.free_reqs.pop_back();
  } else {
    h = (int)s.reqs.size();
    s.reqs.emplace_back();
  }
  s.reqs[h] = Request();
  return h;
}

bool tag_matches(int want, int have) { return want == MPI_ANY_TAG || want == have; }

// Delivers a message into receive request r; lock held.
void deliver(Request& r, const void* data, long bytes, int tag) {
  if (bytes > r.bytes) fatal("message longer than the receive buffer (MPI_ERR_TRUNCATE)");
  if (bytes > 0) memcpy(r.rbuf, data, (size_t)bytes);
  r.complete = true;
  r.status.MPI_SOURCE = 0;
  r.status.MPI_TAG = tag;
  r.status.MPI_ERROR = MPI_SUCCESS;
  r.status.shim_bytes = bytes;
}

// Starts a send of request h (lock held): match a posted receive of the same
// communicator in posting order, else buffer the message.
void start_send(State& s, int h) {
  Request& q = s.reqs[h];
  for (size_t i = 0; i < s.posted_recvs.size(); ++i) {
    Request& r = s.reqs[s.posted_recvs[i]];
    if (r.comm == q.comm && tag_matches(r.tag, q.tag)) {
      deliver(r, q.sbuf, q.bytes, q.tag);
      s.posted_recvs.erase(s.posted_recvs.begin() + (long)i);
      q.complete = true;
      q.status.shim_bytes = q.bytes;
      return;
    }
  }
  Message m;
  m.comm = q.comm;
  m.tag = q.tag;
  m.data.assign((const char*)q.sbuf, (const char*)q.sbuf + q.bytes);
  s.unexpected.push_back(std::move(m));
  q.complete = true;
  q.status.shim_bytes = q.bytes;
}

// Starts a receive of request h (lock held): take the oldest buffered message
// that matches, else post the receive.
void start_recv(State& s, int h) {
  Request& r = s.reqs[h];
  for (auto it = s.unexpected.begin(); it != s.unexpected.end(); ++it) {
    if (it->comm == r.comm && tag_matches(r.tag, it->tag)) {
      deliver(r, it->data.data(), (long)it->data.size(), it->tag);
      s.unexpected.erase(it);
      return;
    }
  }
  s.posted_recvs.push_back(h);
}

int make_p2p(bool send, const void* sbuf, void* rbuf, int count, MPI_Datatype t, int peer, int tag,
             MPI_Comm comm, bool persistent, MPI_Request* request) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  check_comm(s, comm);
  check_peer(peer);
  const long bytes = (long)count * type_of(s, t).extent;
  const int h = new_request(s);
  Request& q = s.reqs[h];
  q.kind = send ? kSend : kRecv;
  q.sbuf = sbuf;
  q.rbuf = rbuf;
  q.bytes = bytes;
  q.comm = comm;
  q.tag = tag;
  q.persistent = persistent;
  *request = h;
  if (peer == MPI_PROC_NULL) {
    q.complete = true;
    q.status.MPI_SOURCE = MPI_PROC_NULL;
    q.status.MPI_TAG = MPI_ANY_TAG;
    q.status.shim_bytes = 0;
    q.kind = kDone;
    return MPI_SUCCESS;
  }
  if (persistent) return MPI_SUCCESS;  // inactive until MPI_Start
  q.active = true;
  if (send)
    start_send(s, h);
  else
    start_recv(s, h);
  return MPI_SUCCESS;
}

// Completes request *h if it can (lock held).  Returns true when complete;
// a finished non-persistent request is freed and *h set to the null handle.
bool try_complete(State& s, MPI_Request* h, MPI_Status* status) {
  if (*h == MPI_REQUEST_NULL) return false;
  if (*h < 0 || *h >= (int)s.reqs.size() || s.reqs[*h].kind == kFree) fatal("invalid request");
  Request& q = s.reqs[*h];
  if (q.persistent && !q.active && q.kind != kDone) return false;
  if (!q.complete) return false;
  if (status != MPI_STATUS_IGNORE) *status = q.status;
  if (q.persistent) {
    q.active = false;
    q.complete = false;
  } else {
    s.reqs[*h].kind = kFree;
    s.free_reqs.push_back(*h);
    *h = MPI_REQUEST_NULL;
  }
  return true;
}

bool is_inactive(State& s, MPI_Request h) {
  if (h == MPI_REQUEST_NULL) return true;
  const Request& q = s.reqs[h];
  return q.persistent && !q.active;
}

// A wait that can never finish (a receive no send will match in this
// one-process world) would hang; it is reported after this long instead.
constexpr double kWaitLimitSeconds = 600.0;

double now_seconds() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

}  // namespace

extern "C" {

int MPI_Init(int*, char***) {
  State& s = st();
  s.initialized = true;
  return MPI_SUCCESS;
}

int MPI_Init_thread(int* argc, char*** argv, int required, int* provided) {
  MPI_Init(argc, argv);
  if (provided) *provided = required;
  return MPI_SUCCESS;
}

int MPI_Initialized(int* flag) {
  *flag = st().initialized;
  return MPI_SUCCESS;
}

int MPI_Finalized(int* flag) {
  *flag = st().finalized;
  return MPI_SUCCESS;
}

int MPI_Finalize(void) {
  st().finalized = true;
  return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm, int errorcode) {
  fflush(stdout);
  fflush(stderr);
  _exit(errorcode == 0 ? 1 : errorcode);
}

int MPI_Query_thread(int* provided) {
  *provided = MPI_THREAD_MULTIPLE;
  return MPI_SUCCESS;
}

int MPI_Is_thread_main(int* flag) {
  *flag = 1;
  return MPI_SUCCESS;
}

int MPI_Get_processor_name(char* name, int* resultlen) {
  if (gethostname(name, MPI_MAX_PROCESSOR_NAME) != 0) strcpy(name, "localhost");
  name[MPI_MAX_PROCESSOR_NAME - 1] = 0;
  *resultlen = (int)strlen(name);
  return MPI_SUCCESS;
}

int MPI_Error_string(int errorcode, char* string, int* resultlen) {
  *resultlen = snprintf(string, MPI_MAX_ERROR_STRING, "MPI error %d", errorcode);
  return MPI_SUCCESS;
}

double MPI_Wtime(void) { return now_seconds(); }

double MPI_Wtick(void) { return 1e-9; }

int MPI_Alloc_mem(MPI_Aint size, MPI_Info, void* baseptr) {
  void* p = nullptr;
  if (posix_memalign(&p, 64, size > 0 ? (size_t)size : 1) != 0) return MPI_ERR_OTHER;
  *(void**)baseptr = p;
  return MPI_SUCCESS;
}

int MPI_Free_mem(void* base) {
  free(base);
  return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int* size) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  check_comm(s, comm);
  *size = 1;
  return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm comm, int* rank) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  check_comm(s, comm);
  *rank = 0;
  return MPI_SUCCESS;
}

int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* newcomm) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  check_comm(s, comm);
  s.comms.push_back(true);
  *newcomm = (int)s.comms.size() - 1;
  return MPI_SUCCESS;
}

int MPI_Comm_split(MPI_Comm comm, int color, int, MPI_Comm* newcomm) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  check_comm(s, comm);
  if (color == MPI_UNDEFINED) {
    *newcomm = MPI_COMM_NULL;
    return MPI_SUCCESS;
  }
  s.comms.push_back(true);
  *newcomm = (int)s.comms.size() - 1;
  return MPI_SUCCESS;
}

int MPI_Comm_free(MPI_Comm* comm) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  check_comm(s, *comm);
  if (*comm > MPI_COMM_SELF) s.comms[*comm] = false;
  *comm = MPI_COMM_NULL;
  return MPI_SUCCESS;
}

int MPI_Comm_set_errhandler(MPI_Comm, MPI_Errhandler) { return MPI_SUCCESS; }

int MPI_Type_contiguous(int count, MPI_Datatype oldtype, MPI_Datatype* newtype) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  const TypeInfo o = type_of(s, oldtype);
  TypeInfo t;
  t.live = true;
  t.size = count * o.size;
  t.lb = o.lb;
  t.extent = count * o.extent;
  t.align = o.align;
  s.types.push_back(t);
  *newtype = (int)s.types.size() - 1;
  return MPI_SUCCESS;
}

int MPI_Type_create_struct(int count, const int blocklengths[], const MPI_Aint displacements[],
                           const MPI_Datatype types[], MPI_Datatype* newtype) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  TypeInfo t;
  t.live = true;
  long lb = 0, ub = 0;
  bool first = true;
  for (int i = 0; i < count; ++i) {
    const TypeInfo& m = type_of(s, types[i]);
    const long lo = displacements[i] + m.lb;
    const long hi = lo + blocklengths[i] * m.extent;
    if (first || lo < lb) lb = lo;
    if (first || hi > ub) ub = hi;
    first = false;
    t.size += blocklengths[i] * m.size;
    if (m.align > t.align) t.align = m.align;
  }
  // The extent is padded to the strictest member alignment, as a C struct
  // of these members is (MPI-3.1 section 4.1.6).
  long ext = ub - lb;
  ext = (ext + t.align - 1) / t.align * t.align;
  t.lb = lb;
  t.extent = ext;
  s.types.push_back(t);
  *newtype = (int)s.types.size() - 1;
  return MPI_SUCCESS;
}

int MPI_Type_create_resized(MPI_Datatype oldtype, MPI_Aint lb, MPI_Aint extent,
                            MPI_Datatype* newtype) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  TypeInfo t = type_of(s, oldtype);
  t.lb = lb;
  t.extent = extent;
  s.types.push_back(t);
  *newtype = (int)s.types.size() - 1;
  return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype* datatype) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  type_of(s, *datatype);
  return MPI_SUCCESS;
}

int MPI_Type_free(MPI_Datatype* datatype) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  type_of(s, *datatype);
  if (*datatype >= MPI_SHIM_FIRST_USER_TYPE) s.types[*datatype].live = false;
  *datatype = MPI_DATATYPE_NULL;
  return MPI_SUCCESS;
}

int MPI_Type_size(MPI_Datatype datatype, int* size) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  *size = (int)type_of(s, datatype).size;
  return MPI_SUCCESS;
}

int MPI_Type_get_extent(MPI_Datatype datatype, MPI_Aint* lb, MPI_Aint* extent) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  const TypeInfo& t = type_of(s, datatype);
  *lb = t.lb;
  *extent = t.extent;
  return MPI_SUCCESS;
}

int MPI_Get_count(const MPI_Status* status, MPI_Datatype datatype, int* count) {
  const long ext = extent_of(datatype);
  if (ext <= 0 || status->shim_bytes % ext != 0)
    *count = MPI_UNDEFINED;
  else
    *count = (int)(status->shim_bytes / ext);
  return MPI_SUCCESS;
}

int MPI_Isend(const void* buf, int count, MPI_Datatype datatype, int dest, int tag, MPI_Comm comm,
              MPI_Request* request) {
  return make_p2p(true, buf, nullptr, count, datatype, dest, tag, comm, false, request);
}

int MPI_Irecv(void* buf, int count, MPI_Datatype datatype, int source, int tag, MPI_Comm comm,
              MPI_Request* request) {
  return make_p2p(false, nullptr, buf, count, datatype, source, tag, comm, false, request);
}

int MPI_Send(const void* buf, int count, MPI_Datatype datatype, int dest, int tag, MPI_Comm comm) {
  MPI_Request r;
  MPI_Isend(buf, count, datatype, dest, tag, comm, &r);
  return MPI_Wait(&r, MPI_STATUS_IGNORE);
}

int MPI_Recv(void* buf, int count, MPI_Datatype datatype, int source, int tag, MPI_Comm comm,
             MPI_Status* status) {
  MPI_Request r;
  MPI_Irecv(buf, count, datatype, source, tag, comm, &r);
  return MPI_Wait(&r, status);
}

int MPI_Sendrecv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void* recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status* status) {
  MPI_Request r[2];
  MPI_Irecv(recvbuf, recvcount, recvtype, source, recvtag, comm, &r[0]);
  MPI_Isend(sendbuf, sendcount, sendtype, dest, sendtag, comm, &r[1]);
  MPI_Wait(&r[1], MPI_STATUS_IGNORE);
  return MPI_Wait(&r[0], status);
}

int MPI_Send_init(const void* buf, int count, MPI_Datatype datatype, int dest, int tag,
                  MPI_Comm comm, MPI_Request* request) {
  return make_p2p(true, buf, nullptr, count, datatype, dest, tag, comm, true, request);
}

int MPI_Recv_init(void* buf, int count, MPI_Datatype datatype, int source, int tag, MPI_Comm comm,
                  MPI_Request* request) {
  return make_p2p(false, nullptr, buf, count, datatype, source, tag, comm, true, request);
}

int MPI_Start(MPI_Request* request) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  if (*request <= 0 || *request >= (int)s.reqs.size()) fatal("invalid request");
  Request& q = s.reqs[*request];
  if (!q.persistent) fatal("MPI_Start on a non-persistent request");
  if (q.kind == kDone) return MPI_SUCCESS;  // MPI_PROC_NULL peer
  if (q.active) fatal("MPI_Start on an active request");
  q.active = true;
  q.complete = false;
  if (q.kind == kSend)
    start_send(s, *request);
  else
    start_recv(s, *request);
  return MPI_SUCCESS;
}

int MPI_Startall(int count, MPI_Request requests[]) {
  for (int i = 0; i < count; ++i) MPI_Start(&requests[i]);
  return MPI_SUCCESS;
}

int MPI_Request_free(MPI_Request* request) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  if (*request == MPI_REQUEST_NULL) return MPI_SUCCESS;
  Request& q = s.reqs[*request];
  for (size_t i = 0; i < s.posted_recvs.size(); ++i)
    if (s.posted_recvs[i] == *request) {
      s.posted_recvs.erase(s.posted_recvs.begin() + (long)i);
      break;
    }
  q.kind = kFree;
  s.free_reqs.push_back(*request);
  *request = MPI_REQUEST_NULL;
  return MPI_SUCCESS;
}

static void empty_status(MPI_Status* status) {
  if (status == MPI_STATUS_IGNORE) return;
  status->MPI_SOURCE = MPI_ANY_SOURCE;
  status->MPI_TAG = MPI_ANY_TAG;
  status->MPI_ERROR = MPI_SUCCESS;
  status->shim_bytes = 0;
}

int MPI_Test(MPI_Request* request, int* flag, MPI_Status* status) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  if (is_inactive(s, *request)) {
    *flag = 1;
    empty_status(status);
    return MPI_SUCCESS;
  }
  *flag = try_complete(s, request, status) ? 1 : 0;
  return MPI_SUCCESS;
}

int MPI_Testany(int count, MPI_Request requests[], int* index, int* flag, MPI_Status* status) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  bool any_active = false;
  for (int i = 0; i < count; ++i) {
    if (is_inactive(s, requests[i])) continue;
    any_active = true;
    if (try_complete(s, &requests[i], status)) {
      *index = i;
      *flag = 1;
      return MPI_SUCCESS;
    }
  }
  *index = MPI_UNDEFINED;
  *flag = any_active ? 0 : 1;
  if (!any_active) empty_status(status);
  return MPI_SUCCESS;
}

int MPI_Testall(int count, MPI_Request requests[], int* flag, MPI_Status statuses[]) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  for (int i = 0; i < count; ++i) {
    if (is_inactive(s, requests[i])) continue;
    const Request& q = s.reqs[requests[i]];
    if (!q.complete) {
      *flag = 0;
      return MPI_SUCCESS;
    }
  }
  for (int i = 0; i < count; ++i) {
    MPI_Status* st_i = statuses == MPI_STATUSES_IGNORE ? MPI_STATUS_IGNORE : &statuses[i];
    if (is_inactive(s, requests[i]))
      empty_status(st_i);
    else
      try_complete(s, &requests[i], st_i);
  }
  *flag = 1;
  return MPI_SUCCESS;
}

int MPI_Testsome(int incount, MPI_Request requests[], int* outcount, int indices[],
                 MPI_Status statuses[]) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  int n = 0;
  bool any_active = false;
  for (int i = 0; i < incount; ++i) {
    if (is_inactive(s, requests[i])) continue;
    any_active = true;
    MPI_Status* st_i = statuses == MPI_STATUSES_IGNORE ? MPI_STATUS_IGNORE : &statuses[n];
    if (try_complete(s, &requests[i], st_i)) indices[n++] = i;
  }
  *outcount = any_active ? n : MPI_UNDEFINED;
  return MPI_SUCCESS;
}

int MPI_Wait(MPI_Request* request, MPI_Status* status) {
  const double t0 = now_seconds();
  for (;;) {
    int flag = 0;
    MPI_Test(request, &flag, status);
    if (flag) return MPI_SUCCESS;
    if (now_seconds() - t0 > kWaitLimitSeconds)
      fatal("MPI_Wait: no matching message in a one-process world");
    sched_yield();
  }
}

int MPI_Waitany(int count, MPI_Request requests[], int* index, MPI_Status* status) {
  const double t0 = now_seconds();
  for (;;) {
    int flag = 0;
    MPI_Testany(count, requests, index, &flag, status);
    if (flag) return MPI_SUCCESS;
    if (now_seconds() - t0 > kWaitLimitSeconds)
      fatal("MPI_Waitany: no matching message in a one-process world");
    sched_yield();
  }
}

int MPI_Waitall(int count, MPI_Request requests[], MPI_Status statuses[]) {
  const double t0 = now_seconds();
  for (;;) {
    int flag = 0;
    MPI_Testall(count, requests, &flag, statuses);
    if (flag) return MPI_SUCCESS;
    if (now_seconds() - t0 > kWaitLimitSeconds)
      fatal("MPI_Waitall: no matching message in a one-process world");
    sched_yield();
  }
}

int MPI_Iprobe(int source, int tag, MPI_Comm comm, int* flag, MPI_Status* status) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  check_comm(s, comm);
  check_peer(source);
  for (const Message& m : s.unexpected)
    if (m.comm == comm && tag_matches(tag, m.tag)) {
      *flag = 1;
      if (status != MPI_STATUS_IGNORE) {
        status->MPI_SOURCE = 0;
        status->MPI_TAG = m.tag;
        status->MPI_ERROR = MPI_SUCCESS;
        status->shim_bytes = (long long)m.data.size();
      }
      return MPI_SUCCESS;
    }
  *flag = 0;
  return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  check_comm(s, comm);
  return MPI_SUCCESS;
}

int MPI_Bcast(void*, int, MPI_Datatype datatype, int root, MPI_Comm) {
  check_root(root);
  extent_of(datatype);
  return MPI_SUCCESS;
}

int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype, MPI_Op,
               int root, MPI_Comm) {
  check_root(root);
  copy_block(recvbuf, sendbuf, count, datatype);
  return MPI_SUCCESS;
}

int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype, MPI_Op,
                  MPI_Comm) {
  copy_block(recvbuf, sendbuf, count, datatype);
  return MPI_SUCCESS;
}

int MPI_Reduce_scatter(const void* sendbuf, void* recvbuf, const int recvcounts[],
                       MPI_Datatype datatype, MPI_Op, MPI_Comm) {
  copy_block(recvbuf, sendbuf, recvcounts[0], datatype);
  return MPI_SUCCESS;
}

int MPI_Reduce_scatter_block(const void* sendbuf, void* recvbuf, int recvcount,
                             MPI_Datatype datatype, MPI_Op, MPI_Comm) {
  copy_block(recvbuf, sendbuf, recvcount, datatype);
  return MPI_SUCCESS;
}

int MPI_Scan(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype, MPI_Op,
             MPI_Comm) {
  copy_block(recvbuf, sendbuf, count, datatype);
  return MPI_SUCCESS;
}

int MPI_Exscan(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) {
  return MPI_SUCCESS;  // rank 0's result is undefined by the standard
}

int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int,
               MPI_Datatype, int root, MPI_Comm) {
  check_root(root);
  copy_block(recvbuf, sendbuf, sendcount, sendtype);
  return MPI_SUCCESS;
}

int MPI_Gatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                const int[], const int displs[], MPI_Datatype recvtype, int root, MPI_Comm) {
  check_root(root);
  if (sendbuf == MPI_IN_PLACE) return MPI_SUCCESS;
  copy_block((char*)recvbuf + (long)displs[0] * extent_of(recvtype), sendbuf, sendcount, sendtype);
  return MPI_SUCCESS;
}

int MPI_Scatter(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int,
                MPI_Datatype, int root, MPI_Comm) {
  check_root(root);
  if (recvbuf == MPI_IN_PLACE) return MPI_SUCCESS;
  copy_block(recvbuf, sendbuf, sendcount, sendtype);
  return MPI_SUCCESS;
}

int MPI_Scatterv(const void* sendbuf, const int sendcounts[], const int displs[],
                 MPI_Datatype sendtype, void* recvbuf, int, MPI_Datatype, int root, MPI_Comm) {
  check_root(root);
  if (recvbuf == MPI_IN_PLACE) return MPI_SUCCESS;
  copy_block(recvbuf, (const char*)sendbuf + (long)displs[0] * extent_of(sendtype), sendcounts[0],
             sendtype);
  return MPI_SUCCESS;
}

int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int,
                  MPI_Datatype, MPI_Comm) {
  copy_block(recvbuf, sendbuf, sendcount, sendtype);
  return MPI_SUCCESS;
}

int MPI_Allgatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                   const int[], const int displs[], MPI_Datatype recvtype, MPI_Comm) {
  if (sendbuf == MPI_IN_PLACE) return MPI_SUCCESS;
  copy_block((char*)recvbuf + (long)displs[0] * extent_of(recvtype), sendbuf, sendcount, sendtype);
  return MPI_SUCCESS;
}

int MPI_Alltoall(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int,
                 MPI_Datatype, MPI_Comm) {
  copy_block(recvbuf, sendbuf, sendcount, sendtype);
  return MPI_SUCCESS;
}

int MPI_Alltoallv(const void* sendbuf, const int sendcounts[], const int sdispls[],
                  MPI_Datatype sendtype, void* recvbuf, const int[], const int rdispls[],
                  MPI_Datatype recvtype, MPI_Comm) {
  if (sendbuf == MPI_IN_PLACE) return MPI_SUCCESS;
  copy_block((char*)recvbuf + (long)rdispls[0] * extent_of(recvtype),
             (const char*)sendbuf + (long)sdispls[0] * extent_of(sendtype), sendcounts[0],
             sendtype);
  return MPI_SUCCESS;
}

int MPI_File_open(MPI_Comm, const char* filename, int amode, MPI_Info, MPI_File* fh) {
  int flags = 0;
  if (amode & MPI_MODE_RDWR)
    flags |= O_RDWR;
  else if (amode & MPI_MODE_WRONLY)
    flags |= O_WRONLY;
  else
    flags |= O_RDONLY;
  if (amode & MPI_MODE_CREATE) flags |= O_CREAT;
  if (amode & MPI_MODE_EXCL) flags |= O_EXCL;
  if (amode & MPI_MODE_APPEND) flags |= O_APPEND;
  const int fd = open(filename, flags, 0644);
  if (fd < 0) return MPI_ERR_OTHER;
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  FileInfo f;
  f.fd = fd;
  f.delete_on_close = (amode & MPI_MODE_DELETE_ON_CLOSE) != 0;
  f.path = filename;
  s.files.push_back(f);
  *fh = (int)s.files.size() - 1;
  return MPI_SUCCESS;
}

static FileInfo& file_of(State& s, MPI_File fh) {
  if (fh <= 0 || fh >= (int)s.files.size() || s.files[fh].fd < 0) fatal("invalid file handle");
  return s.files[fh];
}

int MPI_File_close(MPI_File* fh) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  FileInfo& f = file_of(s, *fh);
  close(f.fd);
  if (f.delete_on_close) unlink(f.path.c_str());
  f.fd = -1;
  *fh = MPI_FILE_NULL;
  return MPI_SUCCESS;
}

int MPI_File_delete(const char* filename, MPI_Info) {
  return unlink(filename) == 0 ? MPI_SUCCESS : MPI_ERR_OTHER;
}

int MPI_File_set_atomicity(MPI_File, int) { return MPI_SUCCESS; }

int MPI_File_set_errhandler(MPI_File, MPI_Errhandler) { return MPI_SUCCESS; }

int MPI_File_set_size(MPI_File fh, MPI_Offset size) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  return ftruncate(file_of(s, fh).fd, (off_t)size) == 0 ? MPI_SUCCESS : MPI_ERR_OTHER;
}

int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype,
                      const char*, MPI_Info) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  FileInfo& f = file_of(s, fh);
  f.disp = disp;
  f.etype_extent = type_of(s, etype).extent;
  return MPI_SUCCESS;
}

// Offsets count etypes of the current view from its displacement.
static int file_io(MPI_File fh, MPI_Offset offset, void* rbuf, const void* wbuf, int count,
                   MPI_Datatype datatype, MPI_Status* status) {
  int fd;
  off_t pos;
  size_t bytes;
  {
    State& s = st();
    std::lock_guard<std::mutex> lk(s.mu);
    FileInfo& f = file_of(s, fh);
    fd = f.fd;
    pos = (off_t)(f.disp + offset * f.etype_extent);
    bytes = (size_t)count * (size_t)type_of(s, datatype).extent;
  }
  size_t done = 0;
  while (done < bytes) {
    ssize_t n = rbuf ? pread(fd, (char*)rbuf + done, bytes - done, pos + (off_t)done)
                     : pwrite(fd, (const char*)wbuf + done, bytes - done, pos + (off_t)done);
    if (n < 0 && errno == EINTR) continue;
    if (n <= 0) break;
    done += (size_t)n;
  }
  if (status != MPI_STATUS_IGNORE) {
    status->MPI_SOURCE = 0;
    status->MPI_TAG = 0;
    status->MPI_ERROR = done == bytes ? MPI_SUCCESS : MPI_ERR_OTHER;
    status->shim_bytes = (long long)done;
  }
  return done == bytes ? MPI_SUCCESS : MPI_ERR_OTHER;
}

int MPI_File_read_at(MPI_File fh, MPI_Offset offset, void* buf, int count, MPI_Datatype datatype,
                     MPI_Status* status) {
  return file_io(fh, offset, buf, nullptr, count, datatype, status);
}

int MPI_File_write_at(MPI_File fh, MPI_Offset offset, const void* buf, int count,
                      MPI_Datatype datatype, MPI_Status* status) {
  return file_io(fh, offset, nullptr, buf, count, datatype, status);
}

// Non-blocking file I/O completes before returning; the request is a
// finished one so that MPI_Wait/Test return at once.
static int done_request(MPI_Request* request, const MPI_Status& status) {
  State& s = st();
  std::lock_guard<std::mutex> lk(s.mu);
  const int h = new_request(s);
  s.reqs[h].kind = kDone;
  s.reqs[h].complete = true;
  s.reqs[h].status = status;
  *request = h;
  return MPI_SUCCESS;
}

int MPI_File_iread_at(MPI_File fh, MPI_Offset offset, void* buf, int count, MPI_Datatype datatype,
                      MPI_Request* request) {
  MPI_Status status;
  const int rc = file_io(fh, offset, buf, nullptr, count, datatype, &status);
  done_request(request, status);
  return rc;
}

int MPI_File_iwrite_at(MPI_File fh, MPI_Offset offset, const void* buf, int count,
                       MPI_Datatype datatype, MPI_Request* request) {
  MPI_Status status;
  const int rc = file_io(fh, offset, nullptr, buf, count, datatype, &status);
  done_request(request, status);
  return rc;
}

}  // extern "C"
