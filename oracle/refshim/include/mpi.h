// Stand-in for the MPI C++ bindings that the reference's src/Parallel/Parallel.cpp calls, for a
// single process (test infrastructure): reductions and gathers copy, broadcasts and barriers
// return, and point-to-point messages (never reached with one process) abort.
#ifndef CAFFE_REFSHIM_MPI_H
#define CAFFE_REFSHIM_MPI_H

namespace MPI {

struct Datatype { int bytes; };
extern const Datatype INT, DOUBLE, CHAR;
struct Op { int kind; };
extern const Op SUM, MIN, MAX;
const int PROC_NULL = -2;

class Request {
public:
    static void Waitall(int, Request*) {}
};

class Intracomm {
public:
    int Get_rank() const { return 0; }
    int Get_size() const { return 1; }
    void Bcast(void*, int, const Datatype&, int) const {}
    void Barrier() const {}
    void Allreduce(const void* in, void* out, int count, const Datatype& t, const Op&) const;
    void Allgather(const void* in, int count, const Datatype& t, void* out, int, const Datatype&) const;
    void Send(const void*, int, const Datatype&, int, int) const;
    void Recv(void*, int, const Datatype&, int, int) const;
    Request Isend(const void*, int, const Datatype&, int, int) const;
    Request Irecv(void*, int, const Datatype&, int, int) const;
};
extern Intracomm COMM_WORLD;

void Init();
void Finalize();

}  // namespace MPI

#endif
