/*
 * Single-rank MPI stand-in (see mpi.h).  Test infrastructure only: it lets
 * the CAC reference compile and run on one core so that its forces, energies
 * and neighbour lists can be used as the oracle.
 *
 * With one rank every collective is a copy, and a message can only be sent
 * to oneself; such messages are buffered in a mailbox and matched to
 * receives by tag.  A receive or wait that can never be satisfied on one
 * rank aborts with a message instead of hanging.
 */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

/* ---------------------------------------------------------------- types */

#define MAX_DERIVED 64
static long derived_size[MAX_DERIVED];
static int nderived = 0;

static long type_size(MPI_Datatype t)
{
  switch (t) {
    case MPI_CHAR: case MPI_BYTE: case MPI_UNSIGNED_CHAR: return 1;
    case MPI_SHORT: return 2;
    case MPI_INT: case MPI_UNSIGNED: case MPI_FLOAT: return 4;
    case MPI_LONG: case MPI_UNSIGNED_LONG: return (long)sizeof(long);
    case MPI_LONG_LONG: case MPI_UNSIGNED_LONG_LONG: return 8;
    case MPI_DOUBLE: return 8;
    case MPI_DOUBLE_INT: return 16;
    case MPI_2INT: return 8;
    case MPI_LONG_DOUBLE: return (long)sizeof(long double);
    default: break;
  }
  if (t >= 100 && t < 100 + nderived) return derived_size[t - 100];
  fprintf(stderr, "mpi_stub: unknown datatype %d\n", t);
  abort();
  return 0;
}

static void copy_buf(const void *src, void *dst, long nbytes)
{
  if (src == MPI_IN_PLACE || src == dst || nbytes <= 0) return;
  memmove(dst, src, (size_t)nbytes);
}

/* ------------------------------------------------------------- lifecycle */

static int initialized = 0;

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; initialized = 1; return MPI_SUCCESS; }
int MPI_Initialized(int *flag) { *flag = initialized; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }

int MPI_Abort(MPI_Comm comm, int errorcode)
{
  (void)comm;
  fflush(stdout);
  fflush(stderr);
  exit(errorcode ? errorcode : 1);
  return MPI_SUCCESS;
}

double MPI_Wtime(void)
{
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return (double)tv.tv_sec + 1.0e-6 * (double)tv.tv_usec;
}

int MPI_Get_version(int *version, int *subversion) { *version = 3; *subversion = 1; return MPI_SUCCESS; }

int MPI_Get_processor_name(char *name, int *resultlen)
{
  strcpy(name, "localhost");
  *resultlen = (int)strlen(name);
  return MPI_SUCCESS;
}

/* --------------------------------------------------------- communicators */

static int next_comm = 16;

int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }

int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm)
{
  (void)comm; (void)key;
  *newcomm = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : next_comm++;
  return MPI_SUCCESS;
}

int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *newcomm) { (void)comm; *newcomm = next_comm++; return MPI_SUCCESS; }
int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }

/* ------------------------------------------------------ datatypes and ops */

int MPI_Type_size(MPI_Datatype datatype, int *size) { *size = (int)type_size(datatype); return MPI_SUCCESS; }

int MPI_Type_contiguous(int count, MPI_Datatype oldtype, MPI_Datatype *newtype)
{
  if (nderived == MAX_DERIVED) {
    fprintf(stderr, "mpi_stub: too many derived datatypes\n");
    abort();
  }
  derived_size[nderived] = (long)count * type_size(oldtype);
  *newtype = 100 + nderived++;
  return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype *datatype) { (void)datatype; return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype *datatype) { *datatype = MPI_DATATYPE_NULL; return MPI_SUCCESS; }

static int next_op = 64;
int MPI_Op_create(MPI_User_function *function, int commute, MPI_Op *op)
{
  (void)function; (void)commute;
  *op = next_op++;
  return MPI_SUCCESS;
}
int MPI_Op_free(MPI_Op *op) { *op = MPI_OP_NULL; return MPI_SUCCESS; }

/* ------------------------------------------------------------ collectives */

int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }

int MPI_Bcast(void *buffer, int count, MPI_Datatype datatype, int root, MPI_Comm comm)
{
  (void)buffer; (void)count; (void)datatype; (void)root; (void)comm;
  return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype datatype, MPI_Op op, MPI_Comm comm)
{
  (void)op; (void)comm;
  copy_buf(sendbuf, recvbuf, count * type_size(datatype));
  return MPI_SUCCESS;
}

int MPI_Reduce(const void *sendbuf, void *recvbuf, int count,
               MPI_Datatype datatype, MPI_Op op, int root, MPI_Comm comm)
{
  (void)op; (void)root; (void)comm;
  copy_buf(sendbuf, recvbuf, count * type_size(datatype));
  return MPI_SUCCESS;
}

int MPI_Scan(const void *sendbuf, void *recvbuf, int count,
             MPI_Datatype datatype, MPI_Op op, MPI_Comm comm)
{
  (void)op; (void)comm;
  copy_buf(sendbuf, recvbuf, count * type_size(datatype));
  return MPI_SUCCESS;
}

int MPI_Reduce_scatter(const void *sendbuf, void *recvbuf, const int *recvcounts,
                       MPI_Datatype datatype, MPI_Op op, MPI_Comm comm)
{
  (void)op; (void)comm;
  copy_buf(sendbuf, recvbuf, recvcounts[0] * type_size(datatype));
  return MPI_SUCCESS;
}

int MPI_Allgather(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                  void *recvbuf, int recvcount, MPI_Datatype recvtype, MPI_Comm comm)
{
  (void)recvcount; (void)recvtype; (void)comm;
  copy_buf(sendbuf, recvbuf, sendcount * type_size(sendtype));
  return MPI_SUCCESS;
}

int MPI_Allgatherv(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                   void *recvbuf, const int *recvcounts, const int *displs,
                   MPI_Datatype recvtype, MPI_Comm comm)
{
  (void)recvcounts; (void)comm;
  copy_buf(sendbuf, (char *)recvbuf + (long)displs[0] * type_size(recvtype),
           sendcount * type_size(sendtype));
  return MPI_SUCCESS;
}

int MPI_Gather(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
               void *recvbuf, int recvcount, MPI_Datatype recvtype, int root,
               MPI_Comm comm)
{
  (void)recvcount; (void)recvtype; (void)root; (void)comm;
  copy_buf(sendbuf, recvbuf, sendcount * type_size(sendtype));
  return MPI_SUCCESS;
}

/* ------------------------------------------------ point-to-point to self */

typedef struct Message {
  int tag;
  long nbytes;
  char *data;
  struct Message *next;
} Message;

static Message *mailbox_head = NULL;
static Message *mailbox_tail = NULL;

#define MAX_REQUESTS 4096
typedef struct {
  int used;
  int is_recv;
  int complete;
  void *buf;
  long capacity;
  int tag;
  long nbytes;
  int recv_tag;
} Request;
static Request requests[MAX_REQUESTS];

static int new_request(void)
{
  for (int i = 0; i < MAX_REQUESTS; i++)
    if (!requests[i].used) {
      memset(&requests[i], 0, sizeof(Request));
      requests[i].used = 1;
      return i;
    }
  fprintf(stderr, "mpi_stub: too many outstanding requests\n");
  abort();
  return -1;
}

static int tag_match(int want, int have) { return want == MPI_ANY_TAG || want == have; }

static void check_self(int rank, const char *what)
{
  if (rank != 0 && rank != MPI_ANY_SOURCE) {
    fprintf(stderr, "mpi_stub: %s with peer rank %d on a one-rank run\n", what, rank);
    abort();
  }
}

static void deliver(Request *r, const void *data, long nbytes, int tag)
{
  if (nbytes > r->capacity) {
    fprintf(stderr, "mpi_stub: message of %ld bytes truncated to %ld\n", nbytes, r->capacity);
    abort();
  }
  memcpy(r->buf, data, (size_t)nbytes);
  r->nbytes = nbytes;
  r->recv_tag = tag;
  r->complete = 1;
}

static void post_send(const void *buf, long nbytes, int tag)
{
  /* match the oldest pending receive with a compatible tag */
  for (int i = 0; i < MAX_REQUESTS; i++) {
    Request *r = &requests[i];
    if (r->used && r->is_recv && !r->complete && tag_match(r->tag, tag)) {
      deliver(r, buf, nbytes, tag);
      return;
    }
  }
  Message *m = (Message *)malloc(sizeof(Message));
  m->tag = tag;
  m->nbytes = nbytes;
  m->data = (char *)malloc(nbytes > 0 ? (size_t)nbytes : 1);
  if (nbytes > 0) memcpy(m->data, buf, (size_t)nbytes);
  m->next = NULL;
  if (mailbox_tail) mailbox_tail->next = m;
  else mailbox_head = m;
  mailbox_tail = m;
}

static int take_message(Request *r)
{
  Message *prev = NULL;
  for (Message *m = mailbox_head; m; prev = m, m = m->next) {
    if (tag_match(r->tag, m->tag)) {
      deliver(r, m->data, m->nbytes, m->tag);
      if (prev) prev->next = m->next;
      else mailbox_head = m->next;
      if (mailbox_tail == m) mailbox_tail = prev;
      free(m->data);
      free(m);
      return 1;
    }
  }
  return 0;
}

int MPI_Send(const void *buf, int count, MPI_Datatype datatype, int dest, int tag, MPI_Comm comm)
{
  (void)comm;
  if (dest == MPI_PROC_NULL) return MPI_SUCCESS;
  check_self(dest, "send");
  post_send(buf, count * type_size(datatype), tag);
  return MPI_SUCCESS;
}

int MPI_Rsend(const void *buf, int count, MPI_Datatype datatype, int dest, int tag, MPI_Comm comm)
{
  return MPI_Send(buf, count, datatype, dest, tag, comm);
}

int MPI_Isend(const void *buf, int count, MPI_Datatype datatype, int dest, int tag,
              MPI_Comm comm, MPI_Request *request)
{
  MPI_Send(buf, count, datatype, dest, tag, comm);
  int id = new_request();
  requests[id].complete = 1;
  *request = id;
  return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype datatype, int source, int tag,
              MPI_Comm comm, MPI_Request *request)
{
  (void)comm;
  if (source == MPI_PROC_NULL) { *request = MPI_REQUEST_NULL; return MPI_SUCCESS; }
  check_self(source, "receive");
  int id = new_request();
  Request *r = &requests[id];
  r->is_recv = 1;
  r->buf = buf;
  r->capacity = count * type_size(datatype);
  r->tag = tag;
  take_message(r);
  *request = id;
  return MPI_SUCCESS;
}

static void fill_status(MPI_Status *status, const Request *r)
{
  if (status == MPI_STATUS_IGNORE) return;
  status->MPI_SOURCE = 0;
  status->MPI_TAG = r->recv_tag;
  status->MPI_ERROR = MPI_SUCCESS;
  status->nbytes = r->nbytes;
}

int MPI_Wait(MPI_Request *request, MPI_Status *status)
{
  if (*request == MPI_REQUEST_NULL) return MPI_SUCCESS;
  Request *r = &requests[*request];
  if (!r->complete && !take_message(r)) {
    fprintf(stderr, "mpi_stub: wait on a receive that no send on this rank satisfies\n");
    abort();
  }
  fill_status(status, r);
  r->used = 0;
  *request = MPI_REQUEST_NULL;
  return MPI_SUCCESS;
}

int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses)
{
  for (int i = 0; i < count; i++)
    MPI_Wait(&reqs[i], statuses == MPI_STATUSES_IGNORE ? MPI_STATUS_IGNORE : &statuses[i]);
  return MPI_SUCCESS;
}

int MPI_Waitany(int count, MPI_Request *reqs, int *index, MPI_Status *status)
{
  for (int i = 0; i < count; i++) {
    if (reqs[i] == MPI_REQUEST_NULL) continue;
    Request *r = &requests[reqs[i]];
    if (r->complete || take_message(r)) {
      *index = i;
      return MPI_Wait(&reqs[i], status);
    }
  }
  for (int i = 0; i < count; i++)
    if (reqs[i] != MPI_REQUEST_NULL) {
      fprintf(stderr, "mpi_stub: waitany with no satisfiable request\n");
      abort();
    }
  *index = MPI_UNDEFINED;
  return MPI_SUCCESS;
}

int MPI_Recv(void *buf, int count, MPI_Datatype datatype, int source, int tag,
             MPI_Comm comm, MPI_Status *status)
{
  MPI_Request req;
  MPI_Irecv(buf, count, datatype, source, tag, comm, &req);
  return MPI_Wait(&req, status);
}

int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest,
                 int sendtag, void *recvbuf, int recvcount, MPI_Datatype recvtype,
                 int source, int recvtag, MPI_Comm comm, MPI_Status *status)
{
  MPI_Request req;
  MPI_Irecv(recvbuf, recvcount, recvtype, source, recvtag, comm, &req);
  MPI_Send(sendbuf, sendcount, sendtype, dest, sendtag, comm);
  return MPI_Wait(&req, status);
}

int MPI_Request_free(MPI_Request *request)
{
  if (*request != MPI_REQUEST_NULL) requests[*request].used = 0;
  *request = MPI_REQUEST_NULL;
  return MPI_SUCCESS;
}

int MPI_Get_count(const MPI_Status *status, MPI_Datatype datatype, int *count)
{
  *count = (int)(status->nbytes / type_size(datatype));
  return MPI_SUCCESS;
}

/* --------------------------------------------------- Cartesian topology */

int MPI_Cart_create(MPI_Comm comm_old, int ndims, const int *dims, const int *periods,
                    int reorder, MPI_Comm *comm_cart)
{
  (void)comm_old; (void)periods; (void)reorder;
  for (int i = 0; i < ndims; i++)
    if (dims[i] != 1) {
      fprintf(stderr, "mpi_stub: processor grid must be 1 in every dimension\n");
      abort();
    }
  *comm_cart = next_comm++;
  return MPI_SUCCESS;
}

int MPI_Cart_get(MPI_Comm comm, int maxdims, int *dims, int *periods, int *coords)
{
  (void)comm;
  for (int i = 0; i < maxdims; i++) {
    dims[i] = 1;
    periods[i] = 1;
    coords[i] = 0;
  }
  return MPI_SUCCESS;
}

int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *rank_source, int *rank_dest)
{
  (void)comm; (void)direction; (void)disp;
  *rank_source = 0;
  *rank_dest = 0;
  return MPI_SUCCESS;
}

int MPI_Cart_rank(MPI_Comm comm, const int *coords, int *rank)
{
  (void)comm; (void)coords;
  *rank = 0;
  return MPI_SUCCESS;
}
