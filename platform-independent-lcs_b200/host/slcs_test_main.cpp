// slcs_test -- script-driven benchmark runner with the reference's script and
// CSV formats (src/main.cpp:16-99, src/test_setup.hpp:170-382).
//
//   slcs_test [script.txt] [out.csv]
//
// Each script line holds key=value options: algorithm, device_type, size_a,
// size_b (default 256), seed_a, seed_b (default: a counter from 1000),
// iterations (default 1); '#' starts a comment.  Inputs are binary strings
// drawn from std::mt19937 (src/test_utility.hpp:8-18).  Each iteration is
// timed around the whole call (host preparation, copies, combing and
// FromStrands, as the reference times it) and written as one CSV line:
// algorithm,device_type,device,size_a,size_b,source_a,source_b,elapsed_ms,hash,speed
// where speed is cells per microsecond.
#include <chrono>
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "algorithm_registry.hpp"
#include "slcs.h"

namespace {

struct Options
{
    std::string algorithm, device_type, file_a, file_b, rng_a, rng_b;
    int size_a = 256, size_b = 256, seed_a = -1, seed_b = -1, iterations = 1;
};

bool parse_int(const std::string &s, int *out)
{
    if (s.empty()) return false;
    char *end = nullptr;
    long v = std::strtol(s.c_str(), &end, 10);
    if (*end != '\0') return false;
    *out = int(v);
    return true;
}

// One script line -> key/value map; words without '=' are ignored.
std::map<std::string, std::string> parse_line(const std::string &line)
{
    std::map<std::string, std::string> kv;
    std::string body = line.substr(0, line.find('#'));
    // allow "key = value" as well as "key=value"
    std::string norm;
    for (size_t i = 0; i < body.size(); ++i) {
        if (body[i] == '=') {
            while (!norm.empty() && (norm.back() == ' ' || norm.back() == '\t')) norm.pop_back();
            norm += '=';
            while (i + 1 < body.size() && (body[i + 1] == ' ' || body[i + 1] == '\t')) ++i;
        } else {
            norm += body[i];
        }
    }
    std::istringstream ss(norm);
    std::string word;
    while (ss >> word) {
        size_t eq = word.find('=');
        if (eq == std::string::npos || eq == 0) continue;
        kv[word.substr(0, eq)] = word.substr(eq + 1);
    }
    return kv;
}

Options to_options(const std::map<std::string, std::string> &kv)
{
    Options o;
    auto get = [&](const char *k) {
        auto it = kv.find(k);
        return it == kv.end() ? std::string() : it->second;
    };
    o.algorithm = get("algorithm");
    o.device_type = get("device_type");
    o.file_a = get("file_a");
    o.file_b = get("file_b");
    o.rng_a = get("rng_a");
    o.rng_b = get("rng_b");
    int v;
    if (parse_int(get("size_a"), &v)) o.size_a = v;
    if (parse_int(get("size_b"), &v)) o.size_b = v;
    if (parse_int(get("seed_a"), &v)) o.seed_a = v;
    if (parse_int(get("seed_b"), &v)) o.seed_b = v;
    if (parse_int(get("iterations"), &v)) o.iterations = v;
    return o;
}

std::vector<int> random_binary(int size, int seed)
{
    std::vector<int> r(size);
    std::mt19937 rng(seed);
    for (int i = 0; i < size; ++i) r[i] = int(rng() & 1);
    return r;
}

} // namespace

int main(int argc, char **argv)
{
    const char *in_name = argc >= 2 ? argv[1] : "test_default.txt";
    const char *out_name = argc >= 3 ? argv[2] : nullptr;
    std::ifstream in(in_name);
    if (!in) {
        std::fprintf(stderr, "Error: cannot read script '%s'\n", in_name);
        return 1;
    }
    FILE *out = out_name ? std::fopen(out_name, "w") : stdout;
    if (!out) {
        std::fprintf(stderr, "Error: cannot write '%s'\n", out_name);
        return 1;
    }
    std::fprintf(out, "algorithm,device_type,device,size_a,size_b,source_a,source_b,elapsed_ms,hash,speed\n");
    LcsAlgorithmRegistry reg;
    int seed_counter = 1000;
    std::string line;
    while (std::getline(in, line)) {
        auto kv = parse_line(line);
        if (kv.empty()) continue;
        Options o = to_options(kv);
        if (o.seed_a == -1) o.seed_a = seed_counter++;
        if (o.seed_b == -1) o.seed_b = seed_counter++;
        auto a = random_binary(o.size_a, o.seed_a);
        auto b = random_binary(o.size_b, o.seed_b);
        LcsInput input(a.data(), int(a.size()), b.data(), int(b.size()));
        auto impl = reg.Get(o.algorithm, o.device_type);
        if (!impl.ok) {
            std::fprintf(stderr, "Error: Unable to find algorithm '%s'\n", o.algorithm.c_str());
            continue;
        }
        char device[256] = "unknown";
        slcs_device_name(impl.queue ? impl.queue->device() : 0, device, sizeof(device));
        for (int it = 0; it < o.iterations; ++it) {
            try {
                auto t0 = std::chrono::steady_clock::now();
                PermutationMatrix perm = impl(input);
                double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
                int64_t hash = perm.hash();
                std::fprintf(out, "%s,%s,%s,%d,%d,", o.algorithm.c_str(), o.device_type.c_str(), device, o.size_a,
                             o.size_b);
                if (!o.file_a.empty()) std::fprintf(out, "%s,", o.file_a.c_str());
                else std::fprintf(out, "%s(%d),", o.rng_a.c_str(), o.seed_a);
                if (!o.file_b.empty()) std::fprintf(out, "%s,", o.file_b.c_str());
                else std::fprintf(out, "%s(%d),", o.rng_b.c_str(), o.seed_b);
                std::fprintf(out, "%f,%" PRId64 ",%f\n", ms, hash, double(int64_t(o.size_a) * o.size_b) / (ms * 1000.0));
            } catch (const std::exception &e) {
                std::fprintf(stderr, "exception: \n>>> %s\n---------------\n", e.what());
            }
        }
        std::fflush(out);
    }
    if (out != stdout) std::fclose(out);
    return 0;
}
