// Fan-out of one output buffer to every registered consumer, each on its own
// thread (the reference's CallbackManager contract, src/core/callback_manager.h).
// invokeAll returns once every consumer has finished with the buffer, so the
// producer may reuse the buffer afterwards (the reference returns at once and
// a third frame can overwrite a buffer a consumer still reads).
#pragma once

#include <condition_variable>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

#include "../../include/ope/iobuffer.h"

namespace ope {

class CallbackManager {
public:
    using CallbackId = int;
    using OutputCallback = std::function<void(const IOBuffer&)>;

    CallbackManager();
    ~CallbackManager();
    CallbackManager(const CallbackManager&) = delete;
    CallbackManager& operator=(const CallbackManager&) = delete;

    CallbackId addCallback(OutputCallback cb);
    bool removeCallback(CallbackId id);
    void clear();
    size_t getCallbackCount() const;
    // Posts `buffer` to every consumer and waits until all have returned.
    void invokeAll(const IOBuffer& buffer);

private:
    struct Consumer;
    mutable std::mutex mu_;
    std::map<CallbackId, std::unique_ptr<Consumer>> consumers_;
    CallbackId next_id_ = 1;
};

}  // namespace ope
