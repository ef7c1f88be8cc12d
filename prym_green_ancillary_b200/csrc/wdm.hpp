// WDM text files (optionally zstd-compressed) as written by the reference's
// save_wdm_file_sym (cuda/wdmfiles.h:153-222) and read by its
// load_wdm_initial_state (:98-149) and by the unchanged bcw rank solver
// (third_party/bcw/src/wdm_files.rs:23-148).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace bw {
namespace wdm {

// libzstd.so.1 loaded at run time (no header or link dependency).
bool zstd_available();

// Writes `text` to `path`, compressed at level 3 when the name ends in .zst or
// .zst.tmp (cuda/zstd_compat.h:55-61), else verbatim.
void write_file(const std::string& path, const std::string& text);

// Reads a file, decompressing it when it starts with the zstd magic bytes.
std::string read_file(const std::string& path);

// Symmetric WDM: header "rows cols p nlen v", the row and column
// preconditioners, v initial vectors, v current vectors (columns of the
// row-major n_cols x v blocks) and v(v+1)/2 sequence lines (columns of the
// packed nlen x v(v+1)/2 upper-triangle buffer).
std::string format_sym(size_t n_rows, size_t n_cols, uint32_t prime, size_t num_v,
                       const std::vector<uint32_t>& row_precond, const std::vector<uint32_t>& col_precond,
                       const std::vector<uint32_t>& initial_rowmajor, const std::vector<uint32_t>& current_rowmajor,
                       const std::vector<uint32_t>& packed_seq, size_t nlen);

struct InitialState {
    size_t rows = 0, cols = 0, nlen = 0, num_v = 0;
    uint32_t prime = 0;
    std::vector<uint32_t> row_precond, col_precond;
    std::vector<uint32_t> initial_rowmajor;   // cols x num_v
};
// load_wdm_initial_state (cuda/wdmfiles.h:98-149).
InitialState read_initial_state(const std::string& path);

}  // namespace wdm
}  // namespace bw
