/* Single-rank stand-in for the MPI API surface the reference's source calls.
 *
 * Test infrastructure only: used to compile the reference's own C++ sources as
 * the FP64 oracle on a machine without an MPI installation. Every rank query
 * answers rank 0 of 1; reductions, gathers and broadcasts over one rank reduce
 * to a copy (or nothing); point-to-point calls are never reached on one rank.
 * Written for this project; it mirrors only the names and signatures of the
 * MPI standard that the reference uses.
 */
#ifndef SMD_ORACLE_MPI_STUB_H
#define SMD_ORACLE_MPI_STUB_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int source, tag, error; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_UNSIGNED 5
#define MPI_DOUBLE 8
#define MPI_SUM 0
#define MPI_MAX_PROCESSOR_NAME 64
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_SUCCESS 0

static inline size_t smd_mpi_size_of(MPI_Datatype t) {
    switch (t) {
        case MPI_CHAR: return 1;
        case MPI_INT: return sizeof(int);
        case MPI_UNSIGNED: return sizeof(unsigned);
        default: return sizeof(double);
    }
}

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Get_processor_name(char *n, int *len) {
    strcpy(n, "localhost"); *len = 9; return 0;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (s != r) memmove(r, s, (size_t)n * smd_mpi_size_of(t));
    return 0;
}
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    if (s != r) memmove(r, s, (size_t)n * smd_mpi_size_of(t));
    return 0;
}
static inline int MPI_Allgather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, MPI_Comm) {
    if (s != r) memmove(r, s, (size_t)n * smd_mpi_size_of(t));
    return 0;
}
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }

#ifdef __cplusplus
/* The few call sites written against the old C++ bindings. */
namespace MPI {
static const int DOUBLE = MPI_DOUBLE;
static const int INT = MPI_INT;
static const int CHAR = MPI_CHAR;
static const int SUM = MPI_SUM;
struct Intracomm {
    int Get_rank() const { return 0; }
    int Get_size() const { return 1; }
    void Barrier() const {}
    void Gather(const void *s, int n, int t, void *r, int, int, int) const {
        if (s != r) memmove(r, s, (size_t)n * smd_mpi_size_of(t));
    }
    void Allreduce(const void *s, void *r, int n, int t, int) const {
        if (s != r) memmove(r, s, (size_t)n * smd_mpi_size_of(t));
    }
    void Bcast(void *, int, int, int) const {}
};
static Intracomm COMM_WORLD;
}  // namespace MPI
#endif

#endif
