// Symbol export of the OCTproEngine-compatible C++ API of the B200 backend.
#ifndef OPE_B200_EXPORT_H
#define OPE_B200_EXPORT_H
#if defined(__GNUC__) || defined(__clang__)
#define OPE_API __attribute__((visibility("default")))
#else
#define OPE_API
#endif
#endif
