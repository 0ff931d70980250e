/* Oracle shim: CRC checksums only feed checkpoint files, which the oracle does
 * not write; process_data accepts every argument and does nothing. */
#pragma once
#include <vector>
#include <map>
#include <string>
#include <boost/serialization/serialization.hpp>
class checksum {
public:
  unsigned long get_value() const { return 0; }
  template <typename... T> void process_data(const T&...) {}
};
