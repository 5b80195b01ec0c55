/*
 * Single-rank stand-in for the MPI interface the reference solver calls.
 *
 * Test infrastructure only: this header lets the reference's unmodified
 * src .cc files compile in a container without MPI.  With one rank every
 * collective is an identity copy.  The call sites it serves are listed in
 * the reference at domain.cc:34-44, fcalculator_workspace.cc:58,
 * initial_condition*.cc (Allreduce), measure_*.cc (Reduce, Bcast, Gather,
 * Gatherv) and main.cc:16-44.
 */
#ifndef SHHD_ORACLE_SHIM_MPI_H
#define SHHD_ORACLE_SHIM_MPI_H

#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_SUCCESS 0

inline std::size_t shim_mpi_type_size(MPI_Datatype t) {
    return t == MPI_DOUBLE ? sizeof(double) : sizeof(int);
}

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }

inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
    std::memmove(recv, send, static_cast<std::size_t>(count) * shim_mpi_type_size(t));
    return MPI_SUCCESS;
}

inline int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    std::memmove(recv, send, static_cast<std::size_t>(count) * shim_mpi_type_size(t));
    return MPI_SUCCESS;
}

inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }

inline int MPI_Gather(const void* send, int scount, MPI_Datatype stype, void* recv, int, MPI_Datatype, int, MPI_Comm) {
    std::memmove(recv, send, static_cast<std::size_t>(scount) * shim_mpi_type_size(stype));
    return MPI_SUCCESS;
}

inline int MPI_Gatherv(const void* send, int scount, MPI_Datatype stype, void* recv, const int*, const int* displs,
                       MPI_Datatype rtype, int, MPI_Comm) {
    char* dst = static_cast<char*>(recv) + static_cast<std::size_t>(displs[0]) * shim_mpi_type_size(rtype);
    std::memmove(dst, send, static_cast<std::size_t>(scount) * shim_mpi_type_size(stype));
    return MPI_SUCCESS;
}

#endif
