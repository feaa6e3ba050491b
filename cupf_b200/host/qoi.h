// qoi.h — quantities of interest of the APT driver, on host argmax maps.
//
// Same names, inputs and outputs as the reference's QOI classes
// (3DgrainMPI/QOI.h:12-48, QOI.cpp): per-grain voxel volumes in first-seen
// order (calculateQoIs), the line-configuration tip / total / extra areas
// (calculateLineQoIs), the tip sampler (sampleHeights) and the junction search
// on the argmax map (searchJunctionsOnImage, line and 3D variants).  Maps are in
// the reference layout (index i + j*fnx + k*fnx*fny).
#pragma once

#include <map>
#include <string>
#include <unordered_map>
#include <vector>

namespace cupf_host {

struct GlobalConstants;  // phase_field.h

struct QoiGrid {
  int fnx = 0, fny = 0, fnz = 0;
  int num_theta = 0;  // NG
  int nts = 0;        // number of QoI frames (frames 0..nts)
  int num_nodes = 0;  // NN (line junction capacity)
};

class QOI {
 public:
  virtual ~QOI() = default;
  virtual void searchJunctionsOnImage(const QoiGrid& g, const int* alpha) = 0;
  void calculateLineQoIs(const QoiGrid& g, int& cur_tip, const int* alpha, int kt, const float* z,
                         const int* loss_area, int move_count);
  void calculateQoIs(const QoiGrid& g, const int* alpha, int kt);
  void sampleHeights(int& cur_tip, const int* alpha, int fnx, int fny, int fnz);

  std::map<std::string, std::vector<int>> mQoIVectorIntData;
  std::map<std::string, std::vector<float>> mQoIVectorFloatData;
  int mNumActiveGrains = 0;
};

class QOILine : public QOI {
 public:
  explicit QOILine(const QoiGrid& g);
  explicit QOILine(const GlobalConstants& params);  // the reference's constructor
  void searchJunctionsOnImage(const QoiGrid& g, const int* alpha) override;
  // The same records from the device's ascending candidate list over the
  // frames' stacked tip layers (cupf_apt_line_junction_candidates).
  void searchJunctionsOnCells(const QoiGrid& g, const int* alpha, const long long* cells,
                              long long ncells);

 private:
  bool lineRecord(const int* layer, int fnx, int j, int i, int* rec) const;
  void storeRecord(int kt, int nframes, size_t& node_cnt, const int* rec);
  int mNumNodeFeatures = 8;
};

class QOI3D : public QOI {
 public:
  explicit QOI3D(const QoiGrid& g);
  explicit QOI3D(const GlobalConstants& params);  // the reference's constructor
  void searchJunctionsOnImage(const QoiGrid& g, const int* alpha) override;
  // The same records from the device's ascending candidate list and per-cell
  // distinct-value counts (cupf_apt_junction_candidates).
  void searchJunctionsOnCells(const QoiGrid& g, const int* alpha, const long long* cells,
                              long long ncells, const unsigned char* distinct);

 private:
  bool junctionRecord(const QoiGrid& g, const int* alpha, long long C,
                      std::unordered_map<int, int>& occur, int* rec) const;
  int mNumNodeFeatures = 9;
};

}  // namespace cupf_host
