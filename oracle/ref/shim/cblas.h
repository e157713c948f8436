/* The reference includes <cblas.h> (core/pch.h:30, precond/FSAI/LU_main.cpp:2) but
 * calls no CBLAS routine on the hot path; this empty header satisfies the include. */
#ifndef ORACLE_SHIM_CBLAS_H
#define ORACLE_SHIM_CBLAS_H
#endif
