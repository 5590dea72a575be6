/* Probe-only MPI declarations so the reference engine header
 * (quad/GPUquad/GPUquad.h, which includes <mpi.h>) compiles without an MPI
 * installation.  The reference calls MPI only when numDevices > 1
 * (GPUquad.h:629-640); the driver always passes numDevices = 1, so none of
 * these functions runs.  Each returns an error code if it ever did. */
#ifndef REF_DRIVER_MPI_STUB_H
#define REF_DRIVER_MPI_STUB_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_DOUBLE 3
#define MPI_MAX_PROCESSOR_NAME 256
static inline int MPI_Init(int*, char***) { return 1; }
static inline int MPI_Finalize(void) { return 1; }
static inline int MPI_Comm_size(MPI_Comm, int* n) { *n = 1; return 1; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 1; }
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return 1; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return 1; }
static inline int MPI_Get_processor_name(char* name, int* len) { name[0] = 0; *len = 0; return 1; }
static inline double MPI_Wtime(void) { return 0.0; }
#endif
