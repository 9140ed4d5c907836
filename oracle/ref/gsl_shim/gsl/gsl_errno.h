/* Stand-in: the reference's solver returns GSL_SUCCESS from its RHS. */
#ifndef ORACLE_GSL_ERRNO_H
#define ORACLE_GSL_ERRNO_H
#define GSL_SUCCESS 0
#endif
