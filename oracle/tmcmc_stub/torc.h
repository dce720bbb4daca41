/* Stand-in for the torc tasking library's header: the statistics call only
 * torc_gettime (defined by the harness). */
#pragma once
double torc_gettime(void);
