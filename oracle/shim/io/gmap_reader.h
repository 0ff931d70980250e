/* Oracle shim: variant_map.h names gmap_reader; the oracle sets cM directly. */
#pragma once
#include <vector>
#include <string>
class gmap_reader {
public:
  std::vector<long int> pos_bp;
  std::vector<double> pos_cm;
  void readGeneticMapFile(const std::string) {}
};
