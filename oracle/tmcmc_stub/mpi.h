/* Stand-in for <mpi.h>: the reference's TMCMC statistics include it through
 * engine_tmcmc.h but call no MPI function (test infrastructure). */
#pragma once
