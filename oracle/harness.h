/* ORACLE harness -- test infrastructure only (see oracle.h). */
#ifndef EXA_ORACLE_HARNESS_H
#define EXA_ORACLE_HARNESS_H
#endif
