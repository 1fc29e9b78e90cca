// 64-byte aligned owned host buffer (the reference's IOBuffer contract).
#include "../../include/ope/iobuffer.h"

#include <cstdlib>
#include <cstring>

namespace ope {

IOBuffer::IOBuffer() : dataPtr(nullptr), sizeInBytes(0), dataType(DataType::UINT8) {}

IOBuffer::~IOBuffer() { releaseMemory(); }

bool IOBuffer::allocateMemory(size_t bytes) {
    releaseMemory();
    if (bytes == 0) return true;
    void* p = nullptr;
    if (posix_memalign(&p, 64, bytes) != 0) return false;
    std::memset(p, 0, bytes);
    dataPtr = p;
    sizeInBytes = bytes;
    return true;
}

void IOBuffer::releaseMemory() {
    std::free(dataPtr);
    dataPtr = nullptr;
    sizeInBytes = 0;
}

void IOBuffer::setDataType(DataType type) { dataType = type; }
IOBuffer::DataType IOBuffer::getDataType() const { return dataType; }
int IOBuffer::getBitDepth() const { return getDataTypeBitDepth(dataType); }
void* IOBuffer::getDataPointer() { return dataPtr; }
const void* IOBuffer::getDataPointer() const { return dataPtr; }
size_t IOBuffer::getSizeInBytes() const { return sizeInBytes; }

}  // namespace ope
