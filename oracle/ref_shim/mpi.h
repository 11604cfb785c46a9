/* Test-infrastructure stub.
 *
 * The reference's headers include <mpi.h> (include/hifde3d/core/environment.hpp)
 * and declare MPI wrappers (include/hifde3d/core/mpi.hpp) that are never
 * called on the factor/apply path. This header supplies only the type names and
 * constants those declarations mention, so the reference's own sources compile
 * without an MPI installation. Nothing here is linked or executed.
 */
#pragma once
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Errhandler;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_ANY_SOURCE -1
#define MPI_ANY_TAG -1
#define MPI_UNDEFINED -32766
#define MPI_COMM_SELF 1
#define MPI_COMM_WORLD 0
#define MPI_ERRORS_RETURN 0
#define MPI_ERRORS_ARE_FATAL 1
#define MPI_REQUEST_NULL 0
#define MPI_MAX 0
#define MPI_MIN 1
#define MPI_MAXLOC 2
#define MPI_MINLOC 3
#define MPI_PROD 4
#define MPI_SUM 5
#define MPI_LAND 6
#define MPI_LOR 7
#define MPI_LXOR 8
#define MPI_BAND 9
#define MPI_BOR 10
#define MPI_BXOR 11
