// Test infrastructure only (oracle build of the reference): a stand-in for
// the reference's HDF5 wrapper (cpp/include/insem/io/hdf5.hpp:14-54), used
// because libhdf5 is not installed on this machine.  Every operation that
// would touch a file throws; the per-step solver path never opens a file, so
// the oracle build of the reference runs its time loop unchanged.
#include <cstdint>
#include <string>
#include <vector>

#include "insem/core/error.hpp"
#include "insem/io/hdf5.hpp"

namespace insem::io {

namespace {
[[noreturn]] void unavailable(const std::string& what) {
  throw Error("HDF5 is not available in the oracle build (" + what + ")");
}
}  // namespace

H5File::H5File(const std::string& path, Mode) : path_(path) { unavailable("open " + path); }
H5File::~H5File() = default;
H5File::H5File(H5File&& other) noexcept : id_(other.id_), path_(std::move(other.path_)) { other.id_ = -1; }
H5File& H5File::operator=(H5File&& other) noexcept {
  id_ = other.id_;
  path_ = std::move(other.path_);
  other.id_ = -1;
  return *this;
}
void H5File::close() noexcept { id_ = -1; }
bool H5File::exists(const std::string& p) const { unavailable("exists " + p); }
void H5File::create_group(const std::string& p) { unavailable("create_group " + p); }

template <class T>
void H5File::write(const std::string& p, const T*, const std::vector<std::size_t>&) {
  unavailable("write " + p);
}
template <class T>
std::vector<T> H5File::read(const std::string& p, std::vector<std::size_t>*) const {
  unavailable("read " + p);
}

template void H5File::write<double>(const std::string&, const double*, const std::vector<std::size_t>&);
template void H5File::write<float>(const std::string&, const float*, const std::vector<std::size_t>&);
template void H5File::write<std::int32_t>(const std::string&, const std::int32_t*, const std::vector<std::size_t>&);
template void H5File::write<std::int64_t>(const std::string&, const std::int64_t*, const std::vector<std::size_t>&);
template std::vector<double> H5File::read<double>(const std::string&, std::vector<std::size_t>*) const;
template std::vector<float> H5File::read<float>(const std::string&, std::vector<std::size_t>*) const;
template std::vector<std::int32_t> H5File::read<std::int32_t>(const std::string&, std::vector<std::size_t>*) const;
template std::vector<std::int64_t> H5File::read<std::int64_t>(const std::string&, std::vector<std::size_t>*) const;

void H5File::set_attribute(const std::string& o, const std::string&, const std::string&) { unavailable(o); }
void H5File::set_attribute(const std::string& o, const std::string&, std::int64_t) { unavailable(o); }
void H5File::set_attribute(const std::string& o, const std::string&, double) { unavailable(o); }
bool H5File::has_attribute(const std::string& o, const std::string&) const { unavailable(o); }
std::string H5File::attribute_string(const std::string& o, const std::string&) const { unavailable(o); }
std::int64_t H5File::attribute_int(const std::string& o, const std::string&) const { unavailable(o); }
double H5File::attribute_double(const std::string& o, const std::string&) const { unavailable(o); }

}  // namespace insem::io
