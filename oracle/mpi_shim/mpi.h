/*
 * Single-rank MPI stand-in used ONLY to compile the reference solver
 * sources into the CPU oracle (test infrastructure, never product code).
 *
 * Every communicator has exactly one rank.  Collectives therefore reduce
 * over one contribution: they copy the send buffer into the receive buffer
 * (nothing at all for MPI_IN_PLACE).  Point-to-point traffic addressed to
 * MPI_PROC_NULL completes immediately; traffic addressed to rank 0 (self)
 * is reported as an error, because a non-periodic single-rank domain never
 * produces it.  Datatype handles encode their byte size so that copies know
 * how many bytes to move; derived contiguous types live in a small table.
 */
#ifndef HFPS_ORACLE_MPI_SHIM_H
#define HFPS_ORACLE_MPI_SHIM_H

#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include <time.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Errhandler;
typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  int count;
} MPI_Status;
typedef void MPI_User_function(void*, void*, int*, MPI_Datatype*);

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_PROC_NULL (-2)
#define MPI_ANY_SOURCE (-1)
#define MPI_REQUEST_NULL 0
#define MPI_OP_NULL 0
#define MPI_DATATYPE_NULL 0
#define MPI_ERRORS_RETURN 1
#define MPI_TAG_UB 1
#define MPI_IDENT 0
#define MPI_CONGRUENT 1
#define MPI_SIMILAR 2
#define MPI_UNEQUAL 3
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)

/* Built-in datatypes: low byte = element size, upper bits = identity. */
#define MPI_CHAR ((1 << 8) | 1)
#define MPI_BYTE ((2 << 8) | 1)
#define MPI_UINT8_T ((3 << 8) | 1)
#define MPI_INT ((4 << 8) | 4)
#define MPI_UNSIGNED ((5 << 8) | 4)
#define MPI_INT32_T ((6 << 8) | 4)
#define MPI_DOUBLE ((7 << 8) | 8)
#define MPI_UINT64_T ((8 << 8) | 8)
#define MPI_UNSIGNED_LONG_LONG ((9 << 8) | 8)
#define MPI_LONG_LONG ((10 << 8) | 8)
#define MPI_INT64_T ((11 << 8) | 8)
#define MPI_UINT32_T ((13 << 8) | 4)
/* struct { double value; int index; }: 12 bytes of data padded to 16. */
#define MPI_DOUBLE_INT ((12 << 8) | 16)

#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_SUM 3
#define MPI_LAND 4
#define MPI_LOR 5
#define MPI_BAND 6
#define MPI_BOR 7
#define MPI_MAXLOC 8
#define MPI_MINLOC 9

/* Derived contiguous types: handle = 0x40000000 | table index. */
#define HFPS_SHIM_DERIVED_BASE 0x40000000
#define HFPS_SHIM_DERIVED_MAX 64
/* Process-wide shim state.  C++17 inline variables give every translation
 * unit the same object (the initialised flag and the derived-type table are
 * written in one source file and read in others). */
#ifdef __cplusplus
#define HFPS_SHIM_STATE inline
#else
#define HFPS_SHIM_STATE static
#endif
HFPS_SHIM_STATE size_t hfps_shim_derived_size[HFPS_SHIM_DERIVED_MAX];
HFPS_SHIM_STATE int hfps_shim_derived_count = 0;
HFPS_SHIM_STATE int hfps_shim_next_comm = 16;
HFPS_SHIM_STATE int hfps_shim_next_op = 16;
HFPS_SHIM_STATE int hfps_shim_initialized = 0;
HFPS_SHIM_STATE int hfps_shim_finalized = 0;
HFPS_SHIM_STATE int hfps_shim_tag_ub = 32767;

static inline size_t hfps_shim_type_size(MPI_Datatype type) {
  if ((type & HFPS_SHIM_DERIVED_BASE) != 0) {
    const int index = type & ~HFPS_SHIM_DERIVED_BASE;
    return (index >= 0 && index < hfps_shim_derived_count)
               ? hfps_shim_derived_size[index]
               : 0u;
  }
  return (size_t)(type & 0xff);
}

static inline int hfps_shim_copy(const void* send, void* receive, int count,
                                 MPI_Datatype type) {
  if (count < 0) return MPI_ERR_OTHER;
  if (send == MPI_IN_PLACE || send == receive || count == 0) return MPI_SUCCESS;
  if (send == NULL || receive == NULL) return MPI_ERR_OTHER;
  memmove(receive, send, (size_t)count * hfps_shim_type_size(type));
  return MPI_SUCCESS;
}

static inline int MPI_Init(int* argc, char*** argv) {
  (void)argc;
  (void)argv;
  hfps_shim_initialized = 1;
  return MPI_SUCCESS;
}
static inline int MPI_Finalize(void) {
  hfps_shim_finalized = 1;
  return MPI_SUCCESS;
}
static inline int MPI_Initialized(int* flag) {
  *flag = hfps_shim_initialized;
  return MPI_SUCCESS;
}
static inline int MPI_Finalized(int* flag) {
  *flag = hfps_shim_finalized;
  return MPI_SUCCESS;
}
static inline double MPI_Wtime(void) {
  struct timespec now;
  clock_gettime(CLOCK_MONOTONIC, &now);
  return (double)now.tv_sec + 1.0e-9 * (double)now.tv_nsec;
}
static inline int MPI_Comm_rank(MPI_Comm comm, int* rank) {
  if (comm == MPI_COMM_NULL) return MPI_ERR_OTHER;
  *rank = 0;
  return MPI_SUCCESS;
}
static inline int MPI_Comm_size(MPI_Comm comm, int* size) {
  if (comm == MPI_COMM_NULL) return MPI_ERR_OTHER;
  *size = 1;
  return MPI_SUCCESS;
}
static inline int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* out) {
  if (comm == MPI_COMM_NULL) return MPI_ERR_OTHER;
  *out = hfps_shim_next_comm++;
  return MPI_SUCCESS;
}
static inline int MPI_Comm_free(MPI_Comm* comm) {
  *comm = MPI_COMM_NULL;
  return MPI_SUCCESS;
}
static inline int MPI_Comm_compare(MPI_Comm left, MPI_Comm right,
                                   int* result) {
  if (left == MPI_COMM_NULL || right == MPI_COMM_NULL) {
    *result = MPI_UNEQUAL;
  } else {
    *result = left == right ? MPI_IDENT : MPI_CONGRUENT;
  }
  return MPI_SUCCESS;
}
static inline int MPI_Comm_set_errhandler(MPI_Comm comm,
                                          MPI_Errhandler handler) {
  (void)comm;
  (void)handler;
  return MPI_SUCCESS;
}
static inline int MPI_Comm_get_attr(MPI_Comm comm, int key, void* value,
                                    int* flag) {
  (void)comm;
  if (key == MPI_TAG_UB) {
    *(int**)value = &hfps_shim_tag_ub;
    *flag = 1;
  } else {
    *flag = 0;
  }
  return MPI_SUCCESS;
}
static inline int MPI_Type_contiguous(int count, MPI_Datatype old,
                                      MPI_Datatype* out) {
  if (count < 0 || hfps_shim_derived_count >= HFPS_SHIM_DERIVED_MAX)
    return MPI_ERR_OTHER;
  hfps_shim_derived_size[hfps_shim_derived_count] =
      (size_t)count * hfps_shim_type_size(old);
  *out = HFPS_SHIM_DERIVED_BASE | hfps_shim_derived_count++;
  return MPI_SUCCESS;
}
static inline int MPI_Type_commit(MPI_Datatype* type) {
  (void)type;
  return MPI_SUCCESS;
}
static inline int MPI_Type_free(MPI_Datatype* type) {
  *type = MPI_DATATYPE_NULL;
  return MPI_SUCCESS;
}
static inline int MPI_Op_create(MPI_User_function* function, int commute,
                                MPI_Op* op) {
  (void)function;
  (void)commute;
  *op = hfps_shim_next_op++;
  return MPI_SUCCESS;
}
static inline int MPI_Op_free(MPI_Op* op) {
  *op = MPI_OP_NULL;
  return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void* send, void* receive, int count,
                                MPI_Datatype type, MPI_Op op, MPI_Comm comm) {
  (void)op;
  if (comm == MPI_COMM_NULL) return MPI_ERR_OTHER;
  return hfps_shim_copy(send, receive, count, type);
}
static inline int MPI_Reduce(const void* send, void* receive, int count,
                             MPI_Datatype type, MPI_Op op, int root,
                             MPI_Comm comm) {
  (void)op;
  if (comm == MPI_COMM_NULL || root != 0) return MPI_ERR_OTHER;
  return hfps_shim_copy(send, receive, count, type);
}
static inline int MPI_Bcast(void* buffer, int count, MPI_Datatype type,
                            int root, MPI_Comm comm) {
  (void)buffer;
  (void)count;
  (void)type;
  return comm == MPI_COMM_NULL || root != 0 ? MPI_ERR_OTHER : MPI_SUCCESS;
}
static inline int MPI_Allgather(const void* send, int send_count,
                                MPI_Datatype send_type, void* receive,
                                int receive_count, MPI_Datatype receive_type,
                                MPI_Comm comm) {
  (void)receive_count;
  (void)receive_type;
  if (comm == MPI_COMM_NULL) return MPI_ERR_OTHER;
  return hfps_shim_copy(send, receive, send_count, send_type);
}
static inline int MPI_Allgatherv(const void* send, int send_count,
                                 MPI_Datatype send_type, void* receive,
                                 const int* receive_counts,
                                 const int* displacements,
                                 MPI_Datatype receive_type, MPI_Comm comm) {
  (void)receive_counts;
  if (comm == MPI_COMM_NULL) return MPI_ERR_OTHER;
  if (send == MPI_IN_PLACE) return MPI_SUCCESS;
  return hfps_shim_copy(
      send,
      (char*)receive + (size_t)displacements[0] *
                           hfps_shim_type_size(receive_type),
      send_count, send_type);
}
static inline int MPI_Alltoall(const void* send, int send_count,
                               MPI_Datatype send_type, void* receive,
                               int receive_count, MPI_Datatype receive_type,
                               MPI_Comm comm) {
  (void)receive_count;
  (void)receive_type;
  if (comm == MPI_COMM_NULL) return MPI_ERR_OTHER;
  return hfps_shim_copy(send, receive, send_count, send_type);
}
static inline int MPI_Alltoallv(const void* send, const int* send_counts,
                                const int* send_displacements,
                                MPI_Datatype send_type, void* receive,
                                const int* receive_counts,
                                const int* receive_displacements,
                                MPI_Datatype receive_type, MPI_Comm comm) {
  (void)receive_counts;
  if (comm == MPI_COMM_NULL) return MPI_ERR_OTHER;
  return hfps_shim_copy(
      (const char*)send +
          (size_t)send_displacements[0] * hfps_shim_type_size(send_type),
      (char*)receive + (size_t)receive_displacements[0] *
                           hfps_shim_type_size(receive_type),
      send_counts[0], send_type);
}
static inline int MPI_Send(const void* buffer, int count, MPI_Datatype type,
                           int destination, int tag, MPI_Comm comm) {
  (void)buffer;
  (void)count;
  (void)type;
  (void)tag;
  (void)comm;
  return destination == MPI_PROC_NULL ? MPI_SUCCESS : MPI_ERR_OTHER;
}
static inline int MPI_Recv(void* buffer, int count, MPI_Datatype type,
                           int source, int tag, MPI_Comm comm,
                           MPI_Status* status) {
  (void)buffer;
  (void)count;
  (void)type;
  (void)tag;
  (void)comm;
  if (status != MPI_STATUS_IGNORE) {
    status->MPI_SOURCE = MPI_PROC_NULL;
    status->MPI_TAG = -1;
    status->MPI_ERROR = MPI_SUCCESS;
    status->count = 0;
  }
  return source == MPI_PROC_NULL ? MPI_SUCCESS : MPI_ERR_OTHER;
}
static inline int MPI_Sendrecv(const void* send, int send_count,
                               MPI_Datatype send_type, int destination,
                               int send_tag, void* receive, int receive_count,
                               MPI_Datatype receive_type, int source,
                               int receive_tag, MPI_Comm comm,
                               MPI_Status* status) {
  (void)receive_count;
  (void)receive_type;
  (void)send_tag;
  (void)receive_tag;
  (void)comm;
  if (status != MPI_STATUS_IGNORE) {
    status->MPI_SOURCE = source;
    status->MPI_TAG = receive_tag;
    status->MPI_ERROR = MPI_SUCCESS;
    status->count = 0;
  }
  if (destination == MPI_PROC_NULL && source == MPI_PROC_NULL)
    return MPI_SUCCESS;
  if (destination == 0 && source == 0)
    return hfps_shim_copy(send, receive, send_count, send_type);
  return MPI_ERR_OTHER;
}
static inline int MPI_Send_init(const void* buffer, int count,
                                MPI_Datatype type, int destination, int tag,
                                MPI_Comm comm, MPI_Request* request) {
  (void)buffer;
  (void)count;
  (void)type;
  (void)tag;
  (void)comm;
  *request = MPI_REQUEST_NULL;
  return destination == MPI_PROC_NULL ? MPI_SUCCESS : MPI_ERR_OTHER;
}
static inline int MPI_Recv_init(void* buffer, int count, MPI_Datatype type,
                                int source, int tag, MPI_Comm comm,
                                MPI_Request* request) {
  (void)buffer;
  (void)count;
  (void)type;
  (void)tag;
  (void)comm;
  *request = MPI_REQUEST_NULL;
  return source == MPI_PROC_NULL ? MPI_SUCCESS : MPI_ERR_OTHER;
}
static inline int MPI_Startall(int count, MPI_Request* requests) {
  (void)count;
  (void)requests;
  return MPI_SUCCESS;
}
static inline int MPI_Waitall(int count, MPI_Request* requests,
                              MPI_Status* statuses) {
  (void)count;
  (void)requests;
  (void)statuses;
  return MPI_SUCCESS;
}
static inline int MPI_Request_free(MPI_Request* request) {
  *request = MPI_REQUEST_NULL;
  return MPI_SUCCESS;
}
static inline int MPI_Cancel(MPI_Request* request) {
  (void)request;
  return MPI_SUCCESS;
}

#ifdef __cplusplus
}
#endif

#endif
