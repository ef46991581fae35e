// Harness-format runner: `solution <point directory>`.
//
// Reads the platform's case layout (manifest.json, point/q.bin, cases/NNNNNN/{a,b}.bin), runs
// fherma_init once, times each fherma_run with a steady clock around the call only (host
// copies in and out included, as the platform's harness measures it, main.cpp:71-73), writes
// out/NNNNNN/c.bin and rewrites out/results.json after every case. A case that throws is
// reported as "crashed" and the run continues. This is this library's own runner; it links
// the same fherma_* entry points any generated harness would.
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

#include "fherma.h"

namespace fs = std::filesystem;

namespace {

std::string read_all(const fs::path& p) {
    std::ifstream f(p, std::ios::binary);
    if (!f) throw std::runtime_error("cannot read " + p.string());
    std::ostringstream s;
    s << f.rdbuf();
    return s.str();
}

double json_number(const std::string& text, const std::string& key) {
    const std::string k = "\"" + key + "\"";
    const size_t at = text.find(k);
    if (at == std::string::npos) throw std::runtime_error("manifest has no " + key);
    const size_t colon = text.find(':', at + k.size());
    return std::strtod(text.c_str() + colon + 1, nullptr);
}

std::vector<uint32_t> read_u32(const fs::path& p, size_t count) {
    const std::string raw = read_all(p);
    if (raw.size() != count * sizeof(uint32_t)) throw std::runtime_error(p.filename().string() + " has the wrong size");
    std::vector<uint32_t> v(count);
    std::memcpy(v.data(), raw.data(), raw.size());
    return v;
}

std::string case_name(size_t i) {
    char buf[16];
    std::snprintf(buf, sizeof buf, "%06zu", i);
    return buf;
}

void write_results(const fs::path& out, double init_s, const std::vector<std::string>& rows) {
    std::ofstream f(out / "results.json");
    char head[64];
    std::snprintf(head, sizeof head, "{\"init_s\":%.9f,\"cases\":[", init_s);
    f << head;
    for (size_t i = 0; i < rows.size(); ++i) f << (i ? "," : "") << rows[i];
    f << "]}";
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::cerr << "usage: solution <point directory>\n";
        return 2;
    }
    const fs::path root = argv[1];
    const std::string manifest = read_all(root / "manifest.json");
    fherma::Point point;
    point.N = uint32_t(json_number(manifest, "N"));
    point.W = uint32_t(json_number(manifest, "W"));
    point.L = uint32_t(json_number(manifest, "L"));
    point.q.shape = {int64_t(point.L)};
    point.q.data = read_u32(root / "point" / "q.bin", point.L);
    const size_t cases = size_t(json_number(manifest, "cases"));
    const fs::path out = root / "out";
    fs::create_directories(out);

    const auto t0 = std::chrono::steady_clock::now();
    void* state = fherma_init(point);
    const double init_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::vector<std::string> rows;
    write_results(out, init_s, rows);
    const size_t count = size_t(point.N) * point.L;
    for (size_t i = 0; i < cases; ++i) {
        const fs::path dir = root / "cases" / case_name(i);
        char row[128];
        try {
            fherma::Inputs in;
            in.a.shape = in.b.shape = {int64_t(point.N), int64_t(point.L)};
            in.a.data = read_u32(dir / "a.bin", count);
            in.b.data = read_u32(dir / "b.bin", count);
            const auto s = std::chrono::steady_clock::now();
            fherma::Outputs res = fherma_run(state, in);
            const double took = std::chrono::duration<double>(std::chrono::steady_clock::now() - s).count();
            const fs::path od = out / case_name(i);
            fs::create_directories(od);
            std::ofstream f(od / "c.bin", std::ios::binary);
            f.write(reinterpret_cast<const char*>(res.c.data.data()), std::streamsize(res.c.data.size() * 4));
            std::snprintf(row, sizeof row, "{\"i\":%zu,\"seconds\":%.9f,\"status\":\"ok\"}", i, took);
        } catch (const std::exception& e) {
            std::snprintf(row, sizeof row, "{\"i\":%zu,\"seconds\":null,\"status\":\"crashed\"}", i);
            std::cerr << "case " << i << ": " << e.what() << "\n";
        }
        rows.emplace_back(row);
        write_results(out, init_s, rows);
    }
    fherma_free(state);
    write_results(out, init_s, rows);
    return 0;
}
