// Minimal stand-in for the Charm++ runtime header so the reference's PINY
// physics files compile serially for the oracle (oracle/_ref).  Project-written.
#ifndef OA_REF_STUB_CHARM_H
#define OA_REF_STUB_CHARM_H
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "pup.h"
inline int CkMyPe() { return 0; }
inline int CkNumPes() { return 1; }
inline void CkExit() { std::exit(1); }
inline void CkAbort(const char* m) { std::fprintf(stderr, "%s\n", m); std::abort(); }
#define CkPrintf std::printf
#define CmiPrintf std::printf
#define CkAssert(x) ((void)0)
#define CmiMemcpy std::memcpy
#define CmiAssert(x) ((void)0)
inline double CmiWallTimer() { return 0.0; }
class CkMigrateMessage {};
class CkCallback {};
#define PUPmarshall(x)
#endif
