// Sample data types of the OCTproEngine API (same enumerators and values as
// the reference's include/types.h:6-19, so existing callers compile unchanged).
#ifndef OPE_B200_TYPES_H
#define OPE_B200_TYPES_H

#include "export.h"

namespace ope {

enum class DataType {
    UINT8 = 1,
    UINT16 = 2,
    UINT32 = 3,
    UINT64 = 4,
    INT8 = 5,
    INT16 = 6,
    INT32 = 7,
    INT64 = 8,
    FLOAT32 = 9,
    FLOAT64 = 10,
    COMPLEX_FLOAT32 = 11,
    COMPLEX_FLOAT64 = 12
};

// Bits and bytes per sample (src/core/types.cpp:5-53 of the reference).
OPE_API int getDataTypeBitDepth(DataType type);
OPE_API int getDataTypeByteSize(DataType type);

}  // namespace ope

#endif
