// Host-side checks of the C++ interface (include/smina_b200.hpp), in the
// manner of the reference's own C++ test programs (src/gpu/tests): settings
// out of range, or that the reference accepts but this engine does not
// build, are refused at construction with std::runtime_error; --fast's
// chain split and step fraction are accepted; device lists parse like the
// reference's parse_devices, and a machine without a usable device gets an
// exception from the constructor instead of a half-built engine.
//
//   gpu_docking_api_test host          (no device present)
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>

#include "smina_b200.hpp"

using smina_b200::GpuDocking;
using smina_b200::GpuSettings;

static int failures = 0;

static void expect(bool ok, const char* what) {
    if (!ok) {
        std::printf("FAIL: %s\n", what);
        failures++;
    }
}

static void expect_throw(const std::function<void()>& f, const char* needle, const char* what) {
    try {
        f();
        std::printf("FAIL: %s (no exception)\n", what);
        failures++;
    } catch (const std::runtime_error& e) {
        if (!std::strstr(e.what(), needle)) {
            std::printf("FAIL: %s (message \"%s\" lacks \"%s\")\n", what, e.what(), needle);
            failures++;
        }
    }
}

static GpuSettings with(const std::function<void(GpuSettings&)>& f) {
    GpuSettings s;
    f(s);
    return s;
}

int main(int argc, char** argv) {
    const std::string mode = argc > 1 ? argv[1] : "host";
    // parse_devices
    expect(smina_b200::parse_devices("0") == std::vector<int>{0}, "parse 0");
    expect(smina_b200::parse_devices("0,1,3") == (std::vector<int>{0, 1, 3}), "parse 0,1,3");
    expect_throw([] { smina_b200::parse_devices(""); }, "bad device list", "empty list");
    expect_throw([] { smina_b200::parse_devices("0,x"); }, "bad device list", "non-numeric device");
    expect_throw([] { smina_b200::parse_devices("1a"); }, "bad device list", "trailing characters");
    expect_throw([] { smina_b200::parse_devices("-1"); }, "bad device list", "negative device");
    // settings this engine does not build
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.chain_split = -1; })); }, "chain_split",
                 "negative chain_split");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.step_fraction = 1.5; })); }, "step_fraction",
                 "step_fraction above 1");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.early_stop = GpuSettings::EARLY_STOP_FULL; })); },
                 "early_stop", "early_stop");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.threads_per_chain = 128; })); }, "threads_per_chain",
                 "threads_per_chain");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.skip_visited = true; })); }, "fp64",
                 "skip_visited without fp64");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.devices.clear(); })); }, "no CUDA device",
                 "no devices");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.devices = {0, 0}; })); }, "given twice",
                 "duplicate device");
    expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.devices = {-2}; })); }, "bad CUDA device",
                 "negative device ordinal");
    if (mode == "host") {
        // without a usable device the constructor throws (cuda_check in the reference)
        expect_throw([] { GpuDocking g(GpuSettings{}); }, "not usable", "no device present");
        expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.chain_split = 0; s.step_fraction = 0; })); },
                     "not usable", "--fast settings pass validation");
        expect_throw([] { GpuDocking g(with([](GpuSettings& s) { s.fp64 = true; })); }, "not usable",
                     "no device present, fp64");
    }
    std::printf("%s: %d failure(s)\n", mode.c_str(), failures);
    return failures ? 1 : 0;
}
