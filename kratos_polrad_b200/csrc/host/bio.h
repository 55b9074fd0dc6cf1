// Binary container of the reference's binary_io (io/binary/binary_io.h:6-32):
//
//   byte 0          is_little_endian | sizeof(size_t)
//   size_t          header size H (bytes before the bulk data)
//   size_t          number of entries N
//   N x {           tag: size_t length + bytes,
//                   size_t size (bytes), char unit size,
//                   size_t offset (from the start of the bulk data) }
//   bulk data       entries back to back
//
// The writer orders the entries by tag (byte-wise), as the reference's
// std::map does, and packs their data in that order (binary_io_base.cpp:
// 89-131), so a file it writes is byte-identical to the reference's for the
// same entries.  The reader accepts any entry order and offsets (the
// reference's Python writer, visual/binary_io.py:150-175, keeps insertion
// order).  Host code only; little-endian hosts with 8-byte size_t.
#pragma once

#include <cstddef>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace kp::bio
{

struct info_t
{
    std::uint64_t size   = 0;    // bytes
    int           u_size = 0;    // bytes per element (1..127)
    std::uint64_t offset = 0;    // from the start of the bulk data
};

// One entry to write: `count` elements of `u_size` bytes at `data`.
struct view_t
{
    const void *  data   = nullptr;
    std::uint64_t count  = 0;
    int           u_size = 0;
};

// Writes the entries (a later entry with the same tag replaces an earlier
// one, as binary_io::base_t::write does).  Throws std::runtime_error.
void write_file( const std::string & path, const std::vector< std::pair< std::string, view_t > > & entries );

// Reads the header; entries in file order.
class reader_t
{
public:
    explicit reader_t( const std::string & path );
    const std::vector< std::pair< std::string, info_t > > & entries(  ) const { return entries_; }
    bool has( const std::string & tag ) const { return index_.count( tag ) != 0; }
    const info_t & info( const std::string & tag ) const;
    // Copies the entry's bytes into dst (at most cap bytes; throws if the
    // entry is larger); returns its size in bytes.
    std::uint64_t read( const std::string & tag, void * dst, std::uint64_t cap ) const;

private:
    std::string path_;
    std::uint64_t header_size_ = 0, file_size_ = 0;
    std::vector< std::pair< std::string, info_t > > entries_;
    std::map< std::string, std::size_t > index_;
};

}   // namespace kp::bio
