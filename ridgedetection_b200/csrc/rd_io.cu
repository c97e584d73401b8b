// rd_io.cu -- cloud files in the reference's two formats (host code).
//
// Text (rd/utils/samples_set.hpp:254-294 and :444-462): one point per line,
// values separated by white space.  The point count is the number of '\n' in
// the file; the dimension is counted on the first line by extracting values
// until the stream reports end of input -- a value that ends the line without
// trailing white space hits end of input as it is read and is not counted, so
// "1 2 3\n" has dimension 2 and "1 2 3 \n" dimension 3, exactly as the
// reference reads them.  Then every non-empty line gives one point: up to
// `dim` values, extra values ignored, missing ones left 0 (the reference leaves
// them unset).  A count of non-empty lines that differs from the count of
// '\n' is an error, as in the reference.
//
// Binary (tests/test_util.hpp:505-551): n * dim raw floats, row-major; the
// file may be longer, never shorter.
#include "../../include/rd_c_api.h"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iterator>
#include <sstream>
#include <string>

namespace rdb {
// rd_capi.cu: stores the message for rd_last_error() and returns s
rd_status report_error(rd_status s, const char* msg);
}  // namespace rdb

namespace {

rd_status io_fail(const char* msg) { return rdb::report_error(RD_ERR_ARG, msg); }

}  // namespace

rd_status rd_text_cloud_shape(const char* path, int64_t* n, int* dim)
{
    if (!path || !n || !dim) return io_fail("null argument");
    std::ifstream f(path);
    if (f.fail()) return io_fail("cannot open the file for reading");
    const int64_t lines = (int64_t)std::count(std::istreambuf_iterator<char>(f),
                                              std::istreambuf_iterator<char>(), '\n');
    f.clear();
    f.seekg(0);
    std::string line;
    std::getline(f, line, '\n');
    std::istringstream iss(line);
    int d = 0;
    for (;;) {
        float v;
        iss >> v;
        if (iss.eof()) break;
        if (iss.fail()) break;
        ++d;
    }
    *n = lines;
    *dim = d;
    return RD_OK;
}

rd_status rd_load_text_cloud(const char* path, float* out, int64_t n, int dim)
{
    if (!path || (!out && n > 0)) return io_fail("null argument");
    if (n < 0 || dim < 1) return io_fail("bad n or dim");
    std::ifstream f(path);
    if (f.fail()) return io_fail("cannot open the file for reading");
    std::fill(out, out + n * (int64_t)dim, 0.0f);
    int64_t index = 0;
    std::string line;
    while (std::getline(f, line, '\n')) {
        if (line.empty()) continue;
        if (index >= n) return io_fail("incorrect points count read");
        std::istringstream iss(line);
        for (int d = 0; d < dim; ++d)
            if (!(iss >> out[index * dim + d])) break;
        ++index;
    }
    if (index != n) return io_fail("incorrect points count read");
    return RD_OK;
}

rd_status rd_load_binary_cloud(const char* path, int64_t n, int dim, float* out)
{
    if (!path || (!out && n > 0)) return io_fail("null argument");
    if (n < 0 || dim < 1) return io_fail("bad n or dim");
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (f.fail()) return io_fail("cannot open the file for reading in binary mode");
    const int64_t size = (int64_t)f.tellg();
    const int64_t want = n * dim * (int64_t)sizeof(float);
    if (size < want) return io_fail("the file is shorter than n * dim floats");
    f.seekg(0);
    f.read(reinterpret_cast<char*>(out), want);
    if (f.fail()) return io_fail("error while reading the file");
    return RD_OK;
}

rd_status rd_save_binary_cloud(const char* path, const float* pts, int64_t n, int dim)
{
    if (!path || (!pts && n > 0)) return io_fail("null argument");
    if (n < 0 || dim < 1) return io_fail("bad n or dim");
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (f.fail()) return io_fail("cannot open the file for writing in binary mode");
    f.write(reinterpret_cast<const char*>(pts), n * dim * (int64_t)sizeof(float));
    if (f.fail()) return io_fail("error while writing the file");
    return RD_OK;
}
