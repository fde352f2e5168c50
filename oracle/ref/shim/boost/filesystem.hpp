/*
 * Stand-in for <boost/filesystem.hpp> used only to compile the reference's
 * I/O sources into the CPU oracle (test infrastructure).  The reference binds
 * a NON-const `directory_entry&` while iterating (src/InputOutput/inputconf.cpp:78),
 * so the iterator here hands out mutable entries; std::filesystem's does not.
 */
#pragma once
#include <filesystem>
#include <string>
#include <vector>
namespace boost { namespace filesystem {
using path = std::filesystem::path;
struct directory_entry {
    std::filesystem::path p;
    const std::filesystem::path& path() const { return p; }
};
class directory_iterator {
public:
    explicit directory_iterator(const std::filesystem::path& dir) {
        for (const auto& e : std::filesystem::directory_iterator(dir)) entries_.push_back({e.path()});
    }
    std::vector<directory_entry>::iterator begin() { return entries_.begin(); }
    std::vector<directory_entry>::iterator end() { return entries_.end(); }
private:
    std::vector<directory_entry> entries_;
};
inline bool create_directory(const std::string& d) {
    std::error_code ec;
    return std::filesystem::create_directory(d, ec);
}
} }
