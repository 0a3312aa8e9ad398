/* Empty stand-in: the reference GPU driver includes <mpi.h> but makes no MPI call. */
#pragma once
