// Drives ope::Processor the way an acquisition program using the OCTproEngine
// C++ API does: configure, initialize, register two consumers, then stream
// frames through getNextAvailableInputBuffer()/process() and collect the
// outputs delivered to the callbacks.
//
//   processor_stream <in.raw> <out.f32> <N> <ascans_per_bscan> <bscans> <frames>
//
// <in.raw> holds <frames> uint16 buffers back to back; the outputs of the
// first consumer are written to <out.f32> in delivery order. Exit code 0 when
// every frame reached both consumers, in submission order.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <mutex>
#include <thread>
#include <vector>

#include "processor.h"

int main(int argc, char** argv) {
    if (argc != 7) {
        std::fprintf(stderr, "usage: %s in.raw out.f32 N ascans bscans frames\n", argv[0]);
        return 2;
    }
    const int n = std::atoi(argv[3]), a = std::atoi(argv[4]), b = std::atoi(argv[5]), frames = std::atoi(argv[6]);
    const size_t in_elems = static_cast<size_t>(n) * a * b;
    const size_t out_elems = static_cast<size_t>(n / 2) * a * b;
    std::vector<uint16_t> raw(in_elems * frames);
    {
        std::ifstream f(argv[1], std::ios::binary);
        f.read(reinterpret_cast<char*>(raw.data()), static_cast<std::streamsize>(raw.size() * 2));
        if (!f) {
            std::fprintf(stderr, "cannot read %s\n", argv[1]);
            return 2;
        }
    }
    try {
        ope::Processor proc(ope::Backend::B200);
        proc.setInputParameters(n, a, b, ope::DataType::UINT16);
        const float res[4] = {0.5f, static_cast<float>(n - 1) - 40.0f, 60.0f, -20.0f};
        proc.setResamplingCoefficients(res);
        proc.enableResampling(true);
        proc.setInterpolationMethod(ope::InterpolationMethod::CUBIC);
        proc.setWindowParameters(ope::WindowType::GAUSS, 0.5f, 0.9f);
        proc.enableWindowing(true);
        const float disp[4] = {0.0f, 0.0f, 2.0f, -1.0f};
        proc.setDispersionCoefficients(disp, 1.0f);
        proc.enableDispersionCompensation(true);
        proc.enableLogScaling(true);
        proc.setGrayscaleRange(20.0f, 90.0f);
        proc.initialize();

        std::vector<float> out(out_elems * frames);
        std::mutex mu;
        std::condition_variable cv;
        int got1 = 0, got2 = 0;
        bool order_ok = true;
        proc.addOutputCallback([&](const ope::IOBuffer& o) {
            if (o.getSizeInBytes() != out_elems * sizeof(float)) order_ok = false;
            std::lock_guard<std::mutex> lk(mu);
            if (got1 < frames) std::memcpy(out.data() + got1 * out_elems, o.getDataPointer(), out_elems * sizeof(float));
            ++got1;
            cv.notify_all();
        });
        proc.addOutputCallback([&](const ope::IOBuffer&) {
            std::lock_guard<std::mutex> lk(mu);
            ++got2;
            cv.notify_all();
        });
        for (int f = 0; f < frames; ++f) {
            ope::IOBuffer& in = proc.getNextAvailableInputBuffer();
            if (in.getSizeInBytes() < in_elems * 2) {
                std::fprintf(stderr, "input buffer too small\n");
                return 1;
            }
            std::memcpy(in.getDataPointer(), raw.data() + f * in_elems, in_elems * 2);
            proc.process(in);
        }
        {
            std::unique_lock<std::mutex> lk(mu);
            if (!cv.wait_for(lk, std::chrono::seconds(60), [&] { return got1 == frames && got2 == frames; })) {
                std::fprintf(stderr, "timeout: %d/%d frames delivered\n", got1, got2);
                return 1;
            }
        }
        proc.cleanup();
        std::ofstream f(argv[2], std::ios::binary);
        f.write(reinterpret_cast<const char*>(out.data()), static_cast<std::streamsize>(out.size() * sizeof(float)));
        if (!order_ok) {
            std::fprintf(stderr, "unexpected output size\n");
            return 1;
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
