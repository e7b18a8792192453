/* TEST INFRASTRUCTURE ONLY. Stand-ins for the FASP solver library's types,
 * so that the reference's LinearSystem and IsoT_FIM declarations compile
 * for the Jacobian-assembly oracle (oracle/jac_harness.cpp). The assembly
 * calls no FASP routine and never touches these members; only their names
 * are needed (FaspSolver.hpp declares solver objects holding them). */
#ifndef OCP_ORACLE_STUB_FASP_H
#define OCP_ORACLE_STUB_FASP_H
typedef struct { int unused; } input_param;
typedef struct { int maxit; } ITS_param;
typedef struct { int unused; } AMG_param;
typedef struct { int unused; } ILU_param;
typedef struct { int unused; } SWZ_param;
typedef struct { int unused; } dCSRmat;
typedef struct { int unused; } dBSRmat;
typedef struct { int unused; } dvector;
typedef struct { int unused; } ivector;
#endif
