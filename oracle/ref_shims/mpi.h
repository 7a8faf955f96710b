/* Single-process stand-in for the MPI calls the reference compiles against (its MPI layer is
 * out of scope: one GPU, one process).  Collectives copy the local buffer; datatypes are
 * represented by their size in bytes.  Test infrastructure for building the reference only. */
#ifndef SBP_REF_MPI_SHIM_H
#define SBP_REF_MPI_SHIM_H
#include <chrono>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef long MPI_Aint;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_IN_PLACE ((void *)1)

inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline double MPI_Wtime() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
inline int MPI_Type_create_struct(int count, const int *blocklengths, const MPI_Aint *displacements,
                                  const MPI_Datatype *types, MPI_Datatype *newtype) {
    long end = 0;
    for (int i = 0; i < count; ++i) {
        long e = displacements[i] + (long)blocklengths[i] * types[i];
        if (e > end) end = e;
    }
    *newtype = (MPI_Datatype)end;
    return 0;
}
inline int MPI_Type_commit(MPI_Datatype *) { return 0; }
inline int MPI_Type_free(MPI_Datatype *) { return 0; }
inline int MPI_Allgather(const void *send, int scount, MPI_Datatype stype, void *recv, int, MPI_Datatype, MPI_Comm) {
    if (send != MPI_IN_PLACE) std::memcpy(recv, send, (size_t)scount * stype);
    return 0;
}
inline int MPI_Allgatherv(const void *send, int scount, MPI_Datatype stype, void *recv, const int *, const int *displs,
                          MPI_Datatype rtype, MPI_Comm) {
    if (send != MPI_IN_PLACE) std::memcpy((char *)recv + (size_t)displs[0] * rtype, send, (size_t)scount * stype);
    return 0;
}
inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
    if (send != MPI_IN_PLACE) std::memcpy(recv, send, (size_t)count * type);
    return 0;
}
#endif
