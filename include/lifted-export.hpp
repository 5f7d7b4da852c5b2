// Export macros of the drop-in C++ API; same names and meaning as the
// reference's src/lifted-export.hpp:1-29, so that code which defines
// LIFTED_SHARED_DEFINE / LIFTED_EXPORTS builds unchanged.
#ifndef LIFTED_DLLEXPORT_H
#define LIFTED_DLLEXPORT_H

#if !defined(LIFTED_SHARED_DEFINE)
#define LIFTED_DLLEXPORT
#define LIFTED_CONTRIB_DLLEXPORT
#define LIFTED_TEST_DLLEXPORT
#else
#ifndef LIFTED_DLLEXPORT
#if defined(_WIN32)
#if defined(LIFTED_EXPORTS)
#define LIFTED_DLLEXPORT __declspec(dllexport)
#else
#define LIFTED_DLLEXPORT __declspec(dllimport)
#endif
#else
#define LIFTED_DLLEXPORT __attribute__((visibility("default")))
#endif
#endif
#endif

#endif  // LIFTED_DLLEXPORT_H
