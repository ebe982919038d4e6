// Per-temperature accumulation of measured quantities and their statistics
// files: the role of the reference's Measure objects (EnergyMeasure,
// OrderParametersMeasure, ...; Accumulate / SaveData / Reset used at
// Pyrochlore.cu:1643-1765, class source absent). Every measurement adds one
// row of `columns` values per temperature; SaveData writes, per temperature
// (ladder order), the temperature, the number of measurements and for every
// column its mean and the standard error of the mean (independent-sample
// estimate; correlated series need blocking, see cudacode_b200/stats.py).
#pragma once

#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

namespace pyro_host {

class Measure {
 public:
  Measure(int n_temperatures, int columns)
      : nT_(n_temperatures), nc_(columns), sum_(nT_ * nc_, 0.0), sum2_(nT_ * nc_, 0.0) {}

  // values[t * columns + c] for temperature slot t (ladder order).
  void Accumulate(const std::vector<double>& values) {
    if ((int)values.size() != nT_ * nc_) throw std::invalid_argument("Measure: row size");
    for (int i = 0; i < nT_ * nc_; ++i) {
      sum_[i] += values[i];
      sum2_[i] += values[i] * values[i];
    }
    ++count_;
  }

  double Mean(int t, int c) const { return count_ ? sum_[t * nc_ + c] / count_ : 0.0; }

  double Error(int t, int c) const {
    if (count_ < 2) return 0.0;
    const double m = Mean(t, c);
    const double var = (sum2_[t * nc_ + c] / count_ - m * m) * count_ / (count_ - 1);
    return std::sqrt(var > 0.0 ? var / count_ : 0.0);
  }

  long long Count() const { return count_; }

  void SaveData(const std::string& path, const std::vector<double>& temperatures,
                const std::string& columns) const {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw std::runtime_error("cannot open " + path);
    std::fprintf(f, "# T n then mean and error of: %s\n", columns.c_str());
    for (int t = 0; t < nT_; ++t) {
      std::fprintf(f, "%.10g %lld", temperatures[t], count_);
      for (int c = 0; c < nc_; ++c) std::fprintf(f, " %.12g %.6g", Mean(t, c), Error(t, c));
      std::fprintf(f, "\n");
    }
    std::fclose(f);
  }

  void Reset() {
    std::fill(sum_.begin(), sum_.end(), 0.0);
    std::fill(sum2_.begin(), sum2_.end(), 0.0);
    count_ = 0;
  }

 private:
  int nT_, nc_;
  std::vector<double> sum_, sum2_;
  long long count_ = 0;
};

}  // namespace pyro_host
