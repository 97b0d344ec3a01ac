// Single-rank MPI used when no MPI installation exists (declared in
// include/mpi_shim/mpi.h).  Every communicator has exactly one rank (0);
// collectives copy the send buffer to the receive buffer.  Communicator
// handles created by dup/split are tracked so that MPI_Comm_free of an
// unknown handle is reported.
#include <mpi.h>

#include <string.h>
#include <unistd.h>

#include <mutex>
#include <set>

namespace {
std::mutex g_mu;
std::set<int> g_comms;
int g_next = 0x44000010;
int g_initialized = 0;
int g_finalized = 0;

bool known(MPI_Comm c) {
  if (c == MPI_COMM_WORLD || c == MPI_COMM_SELF) return true;
  std::lock_guard<std::mutex> lk(g_mu);
  return g_comms.count(c) != 0;
}

MPI_Comm make_comm() {
  std::lock_guard<std::mutex> lk(g_mu);
  int h = g_next++;
  g_comms.insert(h);
  return h;
}

int type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: return 1;
    case MPI_C_BOOL: return 1;
    case MPI_INT: return 4;
    case MPI_FLOAT: return 4;
    case MPI_LONG: return 8;
    case MPI_UNSIGNED_LONG: return 8;
    case MPI_DOUBLE: return 8;
    case MPI_C_COMPLEX: return 8;
    case MPI_C_DOUBLE_COMPLEX: return 16;
    default: return 0;
  }
}
}  // namespace

extern "C" {

int MPI_Init(int*, char***) {
  g_initialized = 1;
  return MPI_SUCCESS;
}
int MPI_Finalize(void) {
  g_finalized = 1;
  return MPI_SUCCESS;
}
int MPI_Initialized(int* flag) {
  if (flag) *flag = g_initialized;
  return MPI_SUCCESS;
}
int MPI_Finalized(int* flag) {
  if (flag) *flag = g_finalized;
  return MPI_SUCCESS;
}
int MPI_Abort(MPI_Comm, int errorcode) { _exit(errorcode); }

int MPI_Comm_rank(MPI_Comm comm, int* rank) {
  if (!known(comm) || !rank) return MPI_ERR_COMM;
  *rank = 0;
  return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm comm, int* size) {
  if (!known(comm) || !size) return MPI_ERR_COMM;
  *size = 1;
  return MPI_SUCCESS;
}
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* newcomm) {
  if (!newcomm) return MPI_ERR_ARG;
  if (!known(comm)) return MPI_ERR_COMM;
  *newcomm = make_comm();
  return MPI_SUCCESS;
}
int MPI_Comm_free(MPI_Comm* comm) {
  if (!comm) return MPI_ERR_ARG;
  if (*comm == MPI_COMM_WORLD || *comm == MPI_COMM_SELF) return MPI_ERR_COMM;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_comms.erase(*comm)) return MPI_ERR_COMM;
  *comm = MPI_COMM_NULL;
  return MPI_SUCCESS;
}
int MPI_Comm_split(MPI_Comm comm, int color, int, MPI_Comm* newcomm) {
  if (!newcomm) return MPI_ERR_ARG;
  if (!known(comm)) return MPI_ERR_COMM;
  *newcomm = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : make_comm();
  return MPI_SUCCESS;
}
int MPI_Comm_split_type(MPI_Comm comm, int, int, MPI_Info, MPI_Comm* newcomm) {
  if (!newcomm) return MPI_ERR_ARG;
  if (!known(comm)) return MPI_ERR_COMM;
  *newcomm = make_comm();
  return MPI_SUCCESS;
}
MPI_Fint MPI_Comm_c2f(MPI_Comm comm) { return (MPI_Fint)comm; }
MPI_Comm MPI_Comm_f2c(MPI_Fint comm) { return (MPI_Comm)comm; }
int MPI_Barrier(MPI_Comm comm) { return known(comm) ? MPI_SUCCESS : MPI_ERR_COMM; }
int MPI_Bcast(void*, int, MPI_Datatype, int root, MPI_Comm comm) {
  if (!known(comm)) return MPI_ERR_COMM;
  return root == 0 ? MPI_SUCCESS : MPI_ERR_ARG;
}
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype, MPI_Op,
                  MPI_Comm comm) {
  if (!known(comm)) return MPI_ERR_COMM;
  if (sendbuf != MPI_IN_PLACE && sendbuf != recvbuf)
    memmove(recvbuf, sendbuf, (size_t)count * (size_t)type_size(datatype));
  return MPI_SUCCESS;
}
int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int,
                  MPI_Datatype, MPI_Comm comm) {
  if (!known(comm)) return MPI_ERR_COMM;
  if (sendbuf != MPI_IN_PLACE && sendbuf != recvbuf)
    memmove(recvbuf, sendbuf, (size_t)sendcount * (size_t)type_size(sendtype));
  return MPI_SUCCESS;
}
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int,
               MPI_Datatype, int root, MPI_Comm comm) {
  if (!known(comm)) return MPI_ERR_COMM;
  if (root != 0) return MPI_ERR_ARG;  // the only rank is 0
  if (sendbuf != MPI_IN_PLACE && sendbuf != recvbuf)
    memmove(recvbuf, sendbuf, (size_t)sendcount * (size_t)type_size(sendtype));
  return MPI_SUCCESS;
}
int MPI_Get_processor_name(char* name, int* resultlen) {
  if (!name || !resultlen) return MPI_ERR_ARG;
  if (gethostname(name, MPI_MAX_PROCESSOR_NAME) != 0) strcpy(name, "localhost");
  name[MPI_MAX_PROCESSOR_NAME - 1] = 0;
  *resultlen = (int)strlen(name);
  return MPI_SUCCESS;
}
int MPI_Error_string(int errorcode, char* string, int* resultlen) {
  const char* s = errorcode == MPI_SUCCESS    ? "MPI_SUCCESS: no errors"
                  : errorcode == MPI_ERR_COMM ? "MPI_ERR_COMM: invalid communicator"
                  : errorcode == MPI_ERR_ARG  ? "MPI_ERR_ARG: invalid argument"
                                              : "MPI_ERR_OTHER: unknown error";
  if (string) {
    strncpy(string, s, MPI_MAX_ERROR_STRING - 1);
    string[MPI_MAX_ERROR_STRING - 1] = 0;
  }
  if (resultlen) *resultlen = (int)strlen(s);
  return MPI_SUCCESS;
}
int MPI_Dims_create(int nnodes, int ndims, int dims[]) {
  if (nnodes != 1 || ndims < 0 || (ndims && !dims)) return MPI_ERR_ARG;
  for (int i = 0; i < ndims; ++i)
    if (dims[i] == 0) dims[i] = 1;
  return MPI_SUCCESS;
}
int MPI_Type_size(MPI_Datatype datatype, int* size) {
  if (!size) return MPI_ERR_ARG;
  *size = type_size(datatype);
  return *size ? MPI_SUCCESS : MPI_ERR_ARG;
}

}  // extern "C"
