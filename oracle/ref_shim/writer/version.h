/* Stand-in for the reference's generated version.h (a CMake template), used
 * ONLY to compile VCFData.cpp into the writer harness of the test oracle. */
#ifndef VERSION_H_
#define VERSION_H_
extern const char *const prog_timestamp;
extern const char *const prog_version;
extern const char *const prog_bugaddress;
#define GIT_BRANCH "harness"
#define GIT_REF "harness"
#endif
