/*
 * Single-rank MPI implementation for the oracle build (test infrastructure).
 *
 * World size is 1.  Collectives reduce over one contribution, so they copy
 * the send buffer into the receive buffer (or do nothing for MPI_IN_PLACE).
 * Point-to-point messages can only be addressed to rank 0 itself; they are
 * matched by communicator and tag in posting order, which is what the
 * reference's CommunicationHelperClass relies on when it moves level
 * permutations through self-messages at np=1
 * (ParGeMSLR SRC/matrices/parallel_csr_matrix.cpp:571-983).
 */
#include "mpi.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <vector>

namespace {

inline size_t dt_size(MPI_Datatype dt) { return (size_t)(dt & 0xff); }

struct Message {
   MPI_Comm comm;
   int tag;
   std::vector<char> data;
};

struct Request {
   bool is_recv;
   bool done;
   void *buf;
   size_t cap_bytes;
   MPI_Comm comm;
   int tag;
   size_t got_bytes;
};

std::deque<Message> g_unexpected;          /* sent, not yet received */
std::map<int, Request> g_requests;          /* live requests by handle */
std::vector<int> g_pending_recv_order;      /* receive handles in posting order */
int g_next_request = 1;
int g_next_comm = 2;
bool g_initialized = false;

bool tag_match(int want, int have) { return want == MPI_ANY_TAG || want == have; }

void fail(const char *what)
{
   std::fprintf(stderr, "mpi_single: %s\n", what);
   std::abort();
}

/* try to complete a posted receive from the unexpected-message queue */
bool try_match_recv(Request &r)
{
   for (auto it = g_unexpected.begin(); it != g_unexpected.end(); ++it)
   {
      if (it->comm == r.comm && tag_match(r.tag, it->tag))
      {
         if (it->data.size() > r.cap_bytes) fail("message truncated");
         if (!it->data.empty()) std::memcpy(r.buf, it->data.data(), it->data.size());
         r.got_bytes = it->data.size();
         r.done = true;
         g_unexpected.erase(it);
         return true;
      }
   }
   return false;
}

void forget_pending(int h)
{
   for (size_t i = 0; i < g_pending_recv_order.size(); i++)
   {
      if (g_pending_recv_order[i] == h)
      {
         g_pending_recv_order.erase(g_pending_recv_order.begin() + i);
         return;
      }
   }
}

void deliver(const void *buf, size_t bytes, int tag, MPI_Comm comm)
{
   /* earliest posted matching receive wins */
   for (size_t i = 0; i < g_pending_recv_order.size(); i++)
   {
      Request &r = g_requests[g_pending_recv_order[i]];
      if (!r.done && r.comm == comm && tag_match(r.tag, tag))
      {
         if (bytes > r.cap_bytes) fail("message truncated");
         if (bytes) std::memcpy(r.buf, buf, bytes);
         r.got_bytes = bytes;
         r.done = true;
         g_pending_recv_order.erase(g_pending_recv_order.begin() + i);
         return;
      }
   }
   Message m;
   m.comm = comm;
   m.tag = tag;
   m.data.assign((const char *)buf, (const char *)buf + bytes);
   g_unexpected.push_back(std::move(m));
}

void fill_status(MPI_Status *st, const Request &r)
{
   if (st)
   {
      st->MPI_SOURCE = 0;
      st->MPI_TAG = r.tag;
      st->MPI_ERROR = MPI_SUCCESS;
      st->count_bytes = (int)r.got_bytes;
   }
}

int complete(MPI_Request *req, MPI_Status *st)
{
   if (*req == MPI_REQUEST_NULL) return MPI_SUCCESS;
   auto it = g_requests.find(*req);
   if (it == g_requests.end()) fail("unknown request");
   Request &r = it->second;
   if (r.is_recv && !r.done && !try_match_recv(r))
   {
      fail("receive can never complete on a single rank (no matching send)");
   }
   if (r.is_recv) forget_pending(*req);
   fill_status(st, r);
   g_requests.erase(it);
   *req = MPI_REQUEST_NULL;
   return MPI_SUCCESS;
}

void copy_bytes(void *dst, const void *src, size_t bytes)
{
   if (src == MPI_IN_PLACE || dst == src || bytes == 0) return;
   std::memmove(dst, src, bytes);
}

} // namespace

extern "C" {

int MPI_Init(int *, char ***) { g_initialized = true; return MPI_SUCCESS; }
int MPI_Finalize(void) { g_initialized = false; return MPI_SUCCESS; }
int MPI_Initialized(int *flag) { *flag = g_initialized ? 1 : 0; return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code) { std::exit(code); }
int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_dup(MPI_Comm, MPI_Comm *newcomm) { *newcomm = g_next_comm++; return MPI_SUCCESS; }
int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm *newcomm) { *newcomm = g_next_comm++; return MPI_SUCCESS; }
int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }

double MPI_Wtime(void)
{
   using namespace std::chrono;
   return duration<double>(steady_clock::now().time_since_epoch()).count();
}

int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op, MPI_Comm)
{
   copy_bytes(recvbuf, sendbuf, (size_t)count * dt_size(dt));
   return MPI_SUCCESS;
}

int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op, int, MPI_Comm)
{
   copy_bytes(recvbuf, sendbuf, (size_t)count * dt_size(dt));
   return MPI_SUCCESS;
}

int MPI_Scan(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op, MPI_Comm)
{
   copy_bytes(recvbuf, sendbuf, (size_t)count * dt_size(dt));
   return MPI_SUCCESS;
}

int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, int, MPI_Datatype, MPI_Comm)
{
   copy_bytes(recvbuf, sendbuf, (size_t)scount * dt_size(sdt));
   return MPI_SUCCESS;
}

int MPI_Allgatherv(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, const int *, const int *displs, MPI_Datatype rdt, MPI_Comm)
{
   if (sendbuf == MPI_IN_PLACE) return MPI_SUCCESS;
   copy_bytes((char *)recvbuf + (size_t)displs[0] * dt_size(rdt), sendbuf, (size_t)scount * dt_size(sdt));
   return MPI_SUCCESS;
}

int MPI_Gather(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, int, MPI_Datatype, int, MPI_Comm)
{
   copy_bytes(recvbuf, sendbuf, (size_t)scount * dt_size(sdt));
   return MPI_SUCCESS;
}

int MPI_Alltoall(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, int, MPI_Datatype, MPI_Comm)
{
   copy_bytes(recvbuf, sendbuf, (size_t)scount * dt_size(sdt));
   return MPI_SUCCESS;
}

int MPI_Alltoallv(const void *sendbuf, const int *scounts, const int *sdispls, MPI_Datatype sdt, void *recvbuf, const int *, const int *rdispls, MPI_Datatype rdt, MPI_Comm)
{
   if (sendbuf == MPI_IN_PLACE) return MPI_SUCCESS;
   copy_bytes((char *)recvbuf + (size_t)rdispls[0] * dt_size(rdt),
              (const char *)sendbuf + (size_t)sdispls[0] * dt_size(sdt),
              (size_t)scounts[0] * dt_size(sdt));
   return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm)
{
   if (dest != 0) fail("send to a rank other than 0");
   deliver(buf, (size_t)count * dt_size(dt), tag, comm);
   return MPI_SUCCESS;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request *req)
{
   MPI_Send(buf, count, dt, dest, tag, comm);
   int h = g_next_request++;
   Request r = {false, true, nullptr, 0, comm, tag, 0};
   g_requests[h] = r;
   *req = h;
   return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm, MPI_Request *req)
{
   if (source != 0 && source != MPI_ANY_SOURCE) fail("receive from a rank other than 0");
   int h = g_next_request++;
   Request r = {true, false, buf, (size_t)count * dt_size(dt), comm, tag, 0};
   if (!try_match_recv(r)) g_pending_recv_order.push_back(h);
   g_requests[h] = r;
   *req = h;
   return MPI_SUCCESS;
}

int MPI_Recv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm, MPI_Status *status)
{
   MPI_Request req;
   MPI_Irecv(buf, count, dt, source, tag, comm, &req);
   return complete(&req, status);
}

int MPI_Sendrecv(const void *sendbuf, int scount, MPI_Datatype sdt, int dest, int stag, void *recvbuf, int rcount, MPI_Datatype rdt, int source, int rtag, MPI_Comm comm, MPI_Status *status)
{
   MPI_Send(sendbuf, scount, sdt, dest, stag, comm);
   return MPI_Recv(recvbuf, rcount, rdt, source, rtag, comm, status);
}

int MPI_Wait(MPI_Request *req, MPI_Status *status) { return complete(req, status); }

int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses)
{
   for (int i = 0; i < count; i++)
   {
      complete(&reqs[i], statuses ? &statuses[i] : MPI_STATUS_IGNORE);
   }
   return MPI_SUCCESS;
}

int MPI_Waitany(int count, MPI_Request *reqs, int *index, MPI_Status *status)
{
   /* prefer a request that is already complete, else the first live one */
   int pick = MPI_UNDEFINED;
   for (int i = 0; i < count && pick == MPI_UNDEFINED; i++)
   {
      if (reqs[i] == MPI_REQUEST_NULL) continue;
      Request &r = g_requests[reqs[i]];
      if (r.done || (r.is_recv && try_match_recv(r))) pick = i;
   }
   for (int i = 0; i < count && pick == MPI_UNDEFINED; i++)
   {
      if (reqs[i] != MPI_REQUEST_NULL) pick = i;
   }
   *index = pick;
   if (pick == MPI_UNDEFINED) return MPI_SUCCESS;
   return complete(&reqs[pick], status);
}

} // extern "C"
