// Host sample buffer of the OCTproEngine API (reference include/iobuffer.h:10-34):
// 64-byte aligned, owned memory, typed by DataType.
#ifndef OPE_B200_IOBUFFER_H
#define OPE_B200_IOBUFFER_H

#include <cstddef>

#include "export.h"
#include "types.h"

namespace ope {

class OPE_API IOBuffer {
public:
    using DataType = ope::DataType;

    IOBuffer();
    ~IOBuffer();
    IOBuffer(const IOBuffer&) = delete;
    IOBuffer& operator=(const IOBuffer&) = delete;

    bool allocateMemory(size_t sizeInBytes);
    void releaseMemory();

    void setDataType(DataType type);
    DataType getDataType() const;
    int getBitDepth() const;

    void* getDataPointer();
    const void* getDataPointer() const;

    size_t getSizeInBytes() const;

private:
    void* dataPtr;
    size_t sizeInBytes;
    DataType dataType;
};

}  // namespace ope

#endif
