/* Placeholder so that headers referring to the test framework resolve; the
 * oracle build never compiles the reference's test files. */
#ifndef PHI_ORACLE_SHIM_GUNIT_H_
#define PHI_ORACLE_SHIM_GUNIT_H_
#endif
