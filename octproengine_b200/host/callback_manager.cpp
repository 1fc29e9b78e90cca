#include "callback_manager.h"

#include <cstdio>
#include <exception>

namespace ope {

namespace {
struct Latch {
    std::mutex mu;
    std::condition_variable cv;
    int remaining;
    explicit Latch(int n) : remaining(n) {}
    void count_down() {
        std::lock_guard<std::mutex> lk(mu);
        if (--remaining == 0) cv.notify_all();
    }
    void wait() {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return remaining == 0; });
    }
};
}  // namespace

struct CallbackManager::Consumer {
    OutputCallback cb;
    std::thread th;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<std::pair<const IOBuffer*, std::shared_ptr<Latch>>> q;
    bool stop = false;

    explicit Consumer(OutputCallback f) : cb(std::move(f)) {
        th = std::thread([this] { run(); });
    }
    void run() {
        while (true) {
            std::pair<const IOBuffer*, std::shared_ptr<Latch>> job;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !q.empty(); });
                if (q.empty()) return;  // stop requested and drained
                job = q.front();
                q.pop_front();
            }
            try {
                cb(*job.first);
            } catch (const std::exception& e) {
                std::fprintf(stderr, "ope: output callback threw: %s\n", e.what());
            } catch (...) {
                std::fprintf(stderr, "ope: output callback threw\n");
            }
            job.second->count_down();
        }
    }
    void post(const IOBuffer* b, std::shared_ptr<Latch> l) {
        {
            std::lock_guard<std::mutex> lk(mu);
            q.emplace_back(b, std::move(l));
        }
        cv.notify_one();
    }
    ~Consumer() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_one();
        if (th.joinable()) th.join();
    }
};

CallbackManager::CallbackManager() = default;

CallbackManager::~CallbackManager() { clear(); }

CallbackManager::CallbackId CallbackManager::addCallback(OutputCallback cb) {
    std::lock_guard<std::mutex> lk(mu_);
    const CallbackId id = next_id_++;
    consumers_[id] = std::make_unique<Consumer>(std::move(cb));
    return id;
}

bool CallbackManager::removeCallback(CallbackId id) {
    std::unique_ptr<Consumer> victim;
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = consumers_.find(id);
        if (it == consumers_.end()) return false;
        victim = std::move(it->second);
        consumers_.erase(it);
    }
    victim.reset();  // joins after the current callback
    return true;
}

void CallbackManager::clear() {
    std::map<CallbackId, std::unique_ptr<Consumer>> all;
    {
        std::lock_guard<std::mutex> lk(mu_);
        all.swap(consumers_);
    }
    all.clear();
}

size_t CallbackManager::getCallbackCount() const {
    std::lock_guard<std::mutex> lk(mu_);
    return consumers_.size();
}

void CallbackManager::invokeAll(const IOBuffer& buffer) {
    std::shared_ptr<Latch> latch;
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (consumers_.empty()) return;
        latch = std::make_shared<Latch>(static_cast<int>(consumers_.size()));
        for (auto& kv : consumers_) kv.second->post(&buffer, latch);
    }
    latch->wait();
}

}  // namespace ope
