// Single-rank stand-in for <mpi.h>, written for this project so that the
// reference's sources (which include <mpi.h> from src/PointCloud.hpp:3 and
// src/Octree.hpp:8 for their datatype helpers) compile without an MPI
// installation. Only the names those headers use are declared; every call is a
// no-op for one rank. Used only by oracle/build_ref.sh.
#pragma once
#include <cstddef>
#include <cstring>

typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef std::ptrdiff_t MPI_Aint;

#define MPI_INT 1
#define MPI_FLOAT 2
#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0

inline int MPI_Type_create_struct(int, const int*, const MPI_Aint*, const MPI_Datatype*, MPI_Datatype* t) {
    *t = 100;
    return MPI_SUCCESS;
}
inline int MPI_Type_create_resized(MPI_Datatype, MPI_Aint, MPI_Aint, MPI_Datatype* t) {
    *t = 101;
    return MPI_SUCCESS;
}
inline int MPI_Type_get_extent(MPI_Datatype, MPI_Aint* lb, MPI_Aint* extent) {
    *lb = 0;
    *extent = 0;
    return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* s) {
    *s = 1;
    return MPI_SUCCESS;
}
inline int MPI_Comm_rank(MPI_Comm, int* r) {
    *r = 0;
    return MPI_SUCCESS;
}
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
