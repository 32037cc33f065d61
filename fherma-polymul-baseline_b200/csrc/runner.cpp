// polymul_solution <point directory>
//
// Point-directory runner in the FHERMA bundle format that the reference's
// harness reads and writes (main.cpp:137-208 there):
//   manifest.json          {"point": {"N": .., "W": .., "L": ..}, "cases": K}
//   point/q.bin            L little-endian u32
//   cases/NNNNNN/a.bin     N x L u32      (and b.bin)
//   out/NNNNNN/c.bin       N x L u32      written
//   out/results.json       {"init_s": s, "cases": [{"i": k, "seconds": s, "status": "ok"}, ...]}
// Only fherma_run is timed.  results.json is rewritten after every case so a
// run cut short keeps what it finished; a case that throws is recorded as
// "crashed" with the message and the run continues.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/fherma_polymul.h"

namespace fs = std::filesystem;

namespace {

std::string read_file(const fs::path& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + path.string());
    std::ostringstream s;
    s << f.rdbuf();
    return s.str();
}

// value of "key": <number> anywhere in a small JSON document
long long json_number(const std::string& doc, const char* key) {
    const std::string pat = std::string("\"") + key + "\"";
    const size_t at = doc.find(pat);
    if (at == std::string::npos) throw std::runtime_error(std::string("manifest.json has no ") + key);
    const size_t colon = doc.find(':', at + pat.size());
    if (colon == std::string::npos) throw std::runtime_error(std::string("manifest.json: bad ") + key);
    return std::strtoll(doc.c_str() + colon + 1, nullptr, 10);
}

std::vector<uint32_t> read_words(const fs::path& path, size_t count) {
    const std::string raw = read_file(path);
    if (raw.size() != count * 4)
        throw std::runtime_error(path.filename().string() + ": " + std::to_string(raw.size()) + " bytes, expected " +
                                 std::to_string(count * 4));
    std::vector<uint32_t> w(count);
    std::memcpy(w.data(), raw.data(), raw.size());
    return w;
}

std::string case_name(size_t i) {
    char buf[32];
    std::snprintf(buf, sizeof buf, "%06zu", i);
    return buf;
}

std::string escape(const std::string& s) {
    std::string out;
    for (char c : s.substr(0, 200)) {
        if (c == '"' || c == '\\') out += '\\';
        out += c == '\n' ? ' ' : c;
    }
    return out;
}

void write_results(const fs::path& out, double init_s, const std::vector<std::string>& cases) {
    std::ofstream f(out / "results.json");
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.9f", init_s);
    f << "{\"init_s\":" << buf << ",\"cases\":[";
    for (size_t i = 0; i < cases.size(); ++i) f << (i ? "," : "") << cases[i];
    f << "]}";
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::cerr << "usage: polymul_solution <point directory>" << std::endl;
        return 2;
    }
    try {
        const fs::path root = argv[1];
        const std::string manifest = read_file(root / "manifest.json");
        fherma::Point p;
        p.N = uint32_t(json_number(manifest, "N"));
        p.W = uint32_t(json_number(manifest, "W"));
        p.L = uint32_t(json_number(manifest, "L"));
        p.q.shape = {int64_t(p.L)};
        p.q.data = read_words(root / "point" / "q.bin", p.L);
        const size_t total = size_t(json_number(manifest, "cases"));
        const fs::path out = root / "out";
        fs::create_directories(out);

        const auto t0 = std::chrono::steady_clock::now();
        void* state = fherma_init(p);
        const double init_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::vector<std::string> results;
        write_results(out, init_s, results);
        const size_t words = size_t(p.N) * p.L;
        for (size_t i = 0; i < total; ++i) {
            const fs::path dir = root / "cases" / case_name(i);
            std::string entry;
            try {
                fherma::Inputs in;
                in.a.shape = in.b.shape = {int64_t(p.N), int64_t(p.L)};
                in.a.data = read_words(dir / "a.bin", words);
                in.b.data = read_words(dir / "b.bin", words);
                const auto s0 = std::chrono::steady_clock::now();
                fherma::Outputs res = fherma_run(state, in);
                const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - s0).count();
                fs::create_directories(out / case_name(i));
                std::ofstream f(out / case_name(i) / "c.bin", std::ios::binary);
                f.write(reinterpret_cast<const char*>(res.c.data.data()), std::streamsize(res.c.data.size() * 4));
                char buf[96];
                std::snprintf(buf, sizeof buf, "{\"i\":%zu,\"seconds\":%.9f,\"status\":\"ok\"}", i, sec);
                entry = buf;
            } catch (const std::exception& e) {
                entry = "{\"i\":" + std::to_string(i) + ",\"seconds\":null,\"status\":\"crashed\",\"note\":\"" +
                        escape(e.what()) + "\"}";
            }
            results.push_back(entry);
            write_results(out, init_s, results);
        }
        fherma_free(state);
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "polymul_solution: " << e.what() << std::endl;
        return 1;
    }
}
