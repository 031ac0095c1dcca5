// Self-test of the single-rank MPI runtime (mpi_shim.cc): the semantics the
// reference driver relies on, checked without the reference.  Prints "ok"
// and exits 0, or names the first failed check and exits 1.
#include <unistd.h>

#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mpi.h"

static int failures = 0;
#define CHECK(c)                                              \
  do {                                                        \
    if (!(c)) {                                               \
      fprintf(stderr, "shim_selftest: %s:%d: %s\n", __FILE__, \
              __LINE__, #c);                                  \
      ++failures;                                             \
    }                                                         \
  } while (0)

struct Edge {  // 12-byte packed record like the reference's edge types
  uint32_t a, b, c;
};
struct Padded {  // long + int: extent padded to 16
  long x;
  int y;
};

int main(int argc, char** argv) {
  int provided = -1;
  MPI_Init_thread(&argc, &argv, MPI_THREAD_FUNNELED, &provided);
  CHECK(provided == MPI_THREAD_FUNNELED);
  int size = 0, rank = -1;
  MPI_Comm_size(MPI_COMM_WORLD, &size);
  MPI_Comm_rank(MPI_COMM_WORLD, &rank);
  CHECK(size == 1 && rank == 0);

  // communicators
  MPI_Comm c1, c2, c3;
  MPI_Comm_split(MPI_COMM_WORLD, 3, 0, &c1);
  MPI_Comm_dup(c1, &c2);
  MPI_Comm_split(MPI_COMM_WORLD, MPI_UNDEFINED, 0, &c3);
  CHECK(c1 != MPI_COMM_NULL && c2 != c1 && c3 == MPI_COMM_NULL);
  MPI_Comm_size(c2, &size);
  CHECK(size == 1);

  // datatypes: contiguous, struct extents, resized
  MPI_Datatype t3, ts, tr;
  MPI_Type_contiguous(3, MPI_UINT32_T, &t3);
  MPI_Type_commit(&t3);
  int tsz = 0;
  MPI_Type_size(t3, &tsz);
  CHECK(tsz == 12);
  int bl[2] = {1, 1};
  MPI_Aint dis[2] = {(MPI_Aint)offsetof(Padded, x), (MPI_Aint)offsetof(Padded, y)};
  MPI_Datatype tys[2] = {MPI_LONG, MPI_INT};
  MPI_Type_create_struct(2, bl, dis, tys, &ts);
  MPI_Aint lb = -1, ext = 0;
  MPI_Type_get_extent(ts, &lb, &ext);
  MPI_Type_size(ts, &tsz);
  CHECK(lb == 0 && ext == (MPI_Aint)sizeof(Padded) && tsz == 12);
  MPI_Type_get_extent(MPI_LONG_INT, &lb, &ext);
  CHECK(ext == (MPI_Aint)sizeof(Padded));
  MPI_Type_create_resized(MPI_INT, 0, 8, &tr);
  MPI_Type_get_extent(tr, &lb, &ext);
  CHECK(ext == 8);

  // collectives copy the caller's own block; MPI_IN_PLACE leaves it
  {
    long s[4] = {1, 2, 3, 4}, r[4] = {0, 0, 0, 0};
    MPI_Allreduce(s, r, 4, MPI_LONG, MPI_SUM, MPI_COMM_WORLD);
    CHECK(memcmp(s, r, sizeof(s)) == 0);
    MPI_Allreduce(MPI_IN_PLACE, r, 4, MPI_LONG, MPI_MAX, MPI_COMM_WORLD);
    CHECK(r[3] == 4);
    std::vector<Edge> send(10), recv(20);
    for (int i = 0; i < 10; ++i) send[i] = Edge{(uint32_t)i, (uint32_t)(2 * i), 7};
    int sc[1] = {6}, sd[1] = {2}, rc[1] = {6}, rd[1] = {5};
    MPI_Alltoallv(send.data(), sc, sd, t3, recv.data(), rc, rd, t3, MPI_COMM_WORLD);
    CHECK(recv[5].a == 2 && recv[10].a == 7 && recv[10].b == 14 && recv[4].a == 0);
    int counts[1] = {3};
    long rs_in[3] = {9, 8, 7}, rs_out[3] = {0, 0, 0};
    MPI_Reduce_scatter(rs_in, rs_out, counts, MPI_LONG, MPI_SUM, MPI_COMM_WORLD);
    CHECK(rs_out[0] == 9 && rs_out[2] == 7);
    int g[4] = {0, 0, 0, 0}, one = 5, displs[1] = {2}, gc[1] = {1};
    MPI_Allgatherv(&one, 1, MPI_INT, g, gc, displs, MPI_INT, MPI_COMM_WORLD);
    CHECK(g[2] == 5 && g[0] == 0);
    Padded pv{42, 3}, po{0, 0};
    MPI_Allreduce(&pv, &po, 1, MPI_LONG_INT, MPI_MAXLOC, MPI_COMM_WORLD);
    CHECK(po.x == 42 && po.y == 3);
  }

  // point to point: receive posted first, then send; send first, then receive
  {
    int a[3] = {1, 2, 3}, b[3] = {0, 0, 0}, c[3] = {0, 0, 0};
    MPI_Request rq[2];
    MPI_Irecv(b, 3, MPI_INT, 0, 11, c1, &rq[0]);
    int flag = 1, idx = -2;
    MPI_Test(&rq[0], &flag, MPI_STATUS_IGNORE);
    CHECK(flag == 0);
    MPI_Isend(a, 2, MPI_INT, 0, 11, c1, &rq[1]);
    MPI_Status st;
    MPI_Testany(2, rq, &idx, &flag, &st);
    CHECK(flag == 1 && idx == 0 && rq[0] == MPI_REQUEST_NULL);
    int got = 0;
    MPI_Get_count(&st, MPI_INT, &got);
    CHECK(got == 2 && b[1] == 2 && st.MPI_TAG == 11);
    MPI_Waitall(2, rq, MPI_STATUSES_IGNORE);
    CHECK(rq[1] == MPI_REQUEST_NULL);
    // tags match, communicators separate
    MPI_Isend(a, 3, MPI_INT, 0, 5, c2, &rq[0]);
    MPI_Irecv(c, 3, MPI_INT, 0, 5, c1, &rq[1]);
    MPI_Test(&rq[1], &flag, MPI_STATUS_IGNORE);
    CHECK(flag == 0);  // the message went to c2
    MPI_Request_free(&rq[1]);
    MPI_Irecv(c, 3, MPI_INT, 0, MPI_ANY_TAG, c2, &rq[1]);
    MPI_Wait(&rq[1], &st);
    CHECK(c[2] == 3 && st.MPI_TAG == 5);
    MPI_Wait(&rq[0], MPI_STATUS_IGNORE);
    // Testany over nothing active reports completion with MPI_UNDEFINED
    MPI_Request none[2] = {MPI_REQUEST_NULL, MPI_REQUEST_NULL};
    MPI_Testany(2, none, &idx, &flag, MPI_STATUS_IGNORE);
    CHECK(flag == 1 && idx == MPI_UNDEFINED);
  }

  // persistent requests can be started again after completion
  {
    int x = 0, y = 0;
    MPI_Request p[2];
    MPI_Send_init(&x, 1, MPI_INT, 0, 9, MPI_COMM_WORLD, &p[0]);
    MPI_Recv_init(&y, 1, MPI_INT, 0, 9, MPI_COMM_WORLD, &p[1]);
    for (int round = 1; round <= 3; ++round) {
      x = 10 * round;
      MPI_Startall(2, p);
      int flag = 0;
      MPI_Testall(2, p, &flag, MPI_STATUSES_IGNORE);
      CHECK(flag == 1 && y == 10 * round && p[0] != MPI_REQUEST_NULL);
    }
    MPI_Request_free(&p[0]);
    MPI_Request_free(&p[1]);
  }

  // files: view displacement in bytes, offsets in etypes
  {
    char path[] = "/tmp/mpi_shim_selftestXXXXXX";
    int fd = mkstemp(path);
    CHECK(fd >= 0);
    close(fd);
    MPI_File fh;
    CHECK(MPI_File_open(MPI_COMM_SELF, path, MPI_MODE_RDWR | MPI_MODE_CREATE | MPI_MODE_DELETE_ON_CLOSE,
                        MPI_INFO_NULL, &fh) == MPI_SUCCESS);
    MPI_File_set_view(fh, 4, t3, t3, "native", MPI_INFO_NULL);
    Edge w[2] = {{1, 2, 3}, {4, 5, 6}}, r[2];
    MPI_File_write_at(fh, 1, w, 2, t3, MPI_STATUS_IGNORE);
    MPI_Request rq;
    MPI_File_iread_at(fh, 1, r, 2, t3, &rq);
    MPI_Wait(&rq, MPI_STATUS_IGNORE);
    CHECK(r[1].c == 6 && r[0].a == 1);
    MPI_File_close(&fh);
    CHECK(access(path, F_OK) != 0);
  }

  MPI_Type_free(&t3);
  MPI_Type_free(&ts);
  MPI_Type_free(&tr);
  MPI_Comm_free(&c1);
  MPI_Comm_free(&c2);
  MPI_Finalize();
  if (failures) return 1;
  printf("ok\n");
  return 0;
}
