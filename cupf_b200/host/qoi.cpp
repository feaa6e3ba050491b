// qoi.cpp — host quantities of interest (see qoi.h).
//
// Algorithms restated from the reference QOI.cpp; the containers whose
// iteration order reaches the output (the std::unordered_map of the junction
// search) are the same standard containers used the same way, so the order of
// the grain ids written per junction is identical for the same C++ library.
// Differences, each a bound the reference lacks: the tip scans stop at the top
// interior layer, ids outside 1..NG are not counted into per-grain arrays, and
// junction lists stop at their preallocated capacity.
#include "qoi.h"

#include <algorithm>
#include <unordered_map>

namespace cupf_host {

static inline bool layer_has_liquid(const int* alpha, int fnx, int fny, int k) {
  const long long off = (long long)fnx * fny * k;
  for (int j = 1; j < fny - 1; ++j)
    for (int i = 1; i < fnx - 1; ++i)
      if (alpha[off + (long long)j * fnx + i] == 0) return true;
  return false;
}

// QOI::sampleHeights (QOI.cpp:162-185): advance to the last fully solid layer.
void QOI::sampleHeights(int& cur_tip, const int* alpha, int fnx, int fny, int fnz) {
  for (;;) {
    cur_tip += 1;
    if (cur_tip >= fnz - 1 || layer_has_liquid(alpha, fnx, fny, cur_tip)) break;
  }
  cur_tip -= 1;
}

QOILine::QOILine(const QoiGrid& g) {
  const int frames = g.nts + 1;
  mQoIVectorFloatData["fractions"] = std::vector<float>((size_t)frames * g.num_theta);
  mQoIVectorIntData["tip_y"] = std::vector<int>(frames);
  mQoIVectorIntData["cross_sec"] = std::vector<int>();
  mQoIVectorIntData["extra_area"] = std::vector<int>((size_t)frames * g.num_theta, 0);
  mQoIVectorIntData["total_area"] = std::vector<int>((size_t)frames * g.num_theta, 0);
  mQoIVectorIntData["tip_final"] = std::vector<int>((size_t)frames * g.num_theta);
  const int repeated_index = 5;
  mQoIVectorIntData["node_region"] =
      std::vector<int>((size_t)frames * repeated_index * g.num_nodes * mNumNodeFeatures, -1);
}

// QOI::calculateLineQoIs (QOI.cpp:38-101)
void QOI::calculateLineQoIs(const QoiGrid& g, int& cur_tip, const int* alpha, int kt,
                            const float* /*z*/, const int* loss_area, int move_count) {
  const int fnx = g.fnx, fny = g.fny, fnz = g.fnz, ng = g.num_theta;
  sampleHeights(cur_tip, alpha, fnx, fny, fnz);
  mQoIVectorIntData["tip_y"][kt] = cur_tip + move_count;
  std::vector<int>& total = mQoIVectorIntData["total_area"];
  std::vector<int>& extra = mQoIVectorIntData["extra_area"];
  for (int k = 1; k < fnz - 1; ++k) {
    const long long off = (long long)fnx * fny * k;
    for (int j = 1; j < fny - 1; ++j)
      for (int i = 1; i < fnx - 1; ++i) {
        const int a = alpha[off + (long long)fnx * j + i];
        if (a > 0 && a <= ng) {
          total[(size_t)kt * ng + a - 1] += 1;
          if (k > cur_tip) extra[(size_t)kt * ng + a - 1] += 1;
        }
      }
  }
  for (int j = 0; j < ng; ++j) total[(size_t)kt * ng + j] += loss_area[j];
}

// The junction record of one cell of a line-configuration cross section, or
// false when its 3x3 in-plane neighbourhood holds fewer than three distinct
// values or one more than five times (the body of the reference's scan,
// QOI.cpp:118-156; a fresh hash map per cell, as there, so the grain ids come
// out in the same order).
bool QOILine::lineRecord(const int* layer, int fnx, int j, int i, int* rec) const {
  std::unordered_map<int, int> occur;
  for (int dj = -1; dj <= 1; ++dj)
    for (int di = -1; di <= 1; ++di) {
      const int v = layer[(long long)(j + dj) * fnx + i + di];
      auto it = occur.find(v);
      if (it != occur.end())
        it->second++;
      else
        occur.insert({v, 1});
    }
  int n_alpha = 0, max_occ = 0;
  for (auto& it : occur) {
    n_alpha++;
    max_occ = std::max(max_occ, it.second);
  }
  if (n_alpha < 3 || max_occ > 5) return false;
  std::fill(rec, rec + mNumNodeFeatures, -1);
  rec[0] = i;
  rec[1] = j;
  rec[2] = max_occ;
  int c = 0;
  for (auto& it : occur)
    if (3 + c < mNumNodeFeatures) rec[3 + c++] = it.first;
  return true;
}

// Stores one record in frame kt's part of node_region (records past the
// frame's preallocated capacity are dropped; the reference writes past it).
// Features the record does not set keep the array's -1.
void QOILine::storeRecord(int kt, int nframes, size_t& node_cnt, const int* rec) {
  std::vector<int>& node = mQoIVectorIntData["node_region"];
  const size_t cap = node.size() / nframes;
  const size_t base = cap * kt;
  if ((node_cnt + 1) * mNumNodeFeatures > cap) return;
  for (int f = 0; f < mNumNodeFeatures; ++f)
    if (rec[f] != -1 || f < 3) node[base + node_cnt * mNumNodeFeatures + f] = rec[f];
  node_cnt++;
}

// QOILine::searchJunctionsOnImage (QOI.cpp:103-160): per saved tip layer, the
// cross section and the 3x3 in-plane neighbourhoods with >= 3 grains.
void QOILine::searchJunctionsOnImage(const QoiGrid& g, const int* alpha) {
  const int fnx = g.fnx, fny = g.fny;
  std::vector<int>& cross = mQoIVectorIntData["cross_sec"];
  const std::vector<int>& tip_y = mQoIVectorIntData["tip_y"];
  int rec[8];
  for (int kt = 0; kt < g.nts + 1; ++kt) {
    const long long off = (long long)fnx * fny * tip_y[kt];
    cross.insert(cross.end(), alpha + off, alpha + off + (long long)fnx * fny);
    size_t node_cnt = 0;
    for (int j = 1; j < fny - 1; ++j)
      for (int i = 1; i < fnx - 1; ++i)
        if (lineRecord(alpha + off, fnx, j, i, rec)) storeRecord(kt, g.nts + 1, node_cnt, rec);
  }
}

// The same records from the device's candidate list: `cells` ascending, each
// an index into the frames' tip layers stacked in frame order
// (kt * fnx * fny + j * fnx + i), as cupf_apt_line_junction_candidates returns
// them.
void QOILine::searchJunctionsOnCells(const QoiGrid& g, const int* alpha, const long long* cells,
                                     long long ncells) {
  const int fnx = g.fnx, fny = g.fny;
  const long long plane = (long long)fnx * fny;
  std::vector<int>& cross = mQoIVectorIntData["cross_sec"];
  const std::vector<int>& tip_y = mQoIVectorIntData["tip_y"];
  int rec[8];
  long long n = 0;
  for (int kt = 0; kt < g.nts + 1; ++kt) {
    const long long off = plane * tip_y[kt];
    cross.insert(cross.end(), alpha + off, alpha + off + plane);
    size_t node_cnt = 0;
    for (; n < ncells && cells[n] / plane == kt; ++n) {
      const int j = (int)((cells[n] % plane) / fnx), i = (int)(cells[n] % fnx);
      if (lineRecord(alpha + off, fnx, j, i, rec)) storeRecord(kt, g.nts + 1, node_cnt, rec);
    }
  }
}

QOI3D::QOI3D(const QoiGrid&) {
  mQoIVectorIntData["volume"] = std::vector<int>();
  mQoIVectorIntData["grainToPF"] = std::vector<int>();
  mQoIVectorIntData["node_region"] = std::vector<int>();
  mQoIVectorIntData["manifold"] = std::vector<int>();
  mQoIVectorFloatData["geodesic_y_coors"] = std::vector<float>();
}

// QOI::calculateQoIs (QOI.cpp:198-231): voxel count of every grain id > 0 over
// the interior, grains listed in order of first occurrence in (k, j, i) order.
void QOI::calculateQoIs(const QoiGrid& g, const int* alpha, int /*kt*/) {
  std::vector<int>& vol = mQoIVectorIntData["volume"];
  std::vector<int>& g2p = mQoIVectorIntData["grainToPF"];
  vol.clear();
  g2p.clear();
  std::unordered_map<int, int> index;
  mNumActiveGrains = 0;
  for (int k = 1; k < g.fnz - 1; ++k) {
    const long long off = (long long)g.fnx * g.fny * k;
    for (int j = 1; j < g.fny - 1; ++j)
      for (int i = 1; i < g.fnx - 1; ++i) {
        const int a = alpha[off + (long long)g.fnx * j + i];
        if (a <= 0) continue;
        auto it = index.find(a);
        if (it == index.end()) {
          it = index.insert({a, mNumActiveGrains++}).first;
          g2p.push_back(a);
          vol.push_back(0);
        }
        vol[it->second] += 1;
      }
  }
}

// QOI3D::searchJunctionsOnImage (QOI.cpp:233-311): solid cells whose
// 19-point neighbourhood (|d|^2 <= 2) holds no liquid and exactly 4 grains.
// The junction record of one cell, or false when the cell is not a junction of
// four grains (the body of the reference's scan, QOI.cpp:244-305).
bool QOI3D::junctionRecord(const QoiGrid& g, const int* alpha, long long C,
                           std::unordered_map<int, int>& occur, int* rec) const {
  const int fnx = g.fnx, fny = g.fny;
  if (alpha[C] == 0) return false;
  occur.clear();
  int zeros = 0;
  for (int dk = -1; dk <= 1; ++dk)
    for (int dj = -1; dj <= 1; ++dj)
      for (int di = -1; di <= 1; ++di) {
        if (di * di + dj * dj + dk * dk > 2) continue;
        const int v = alpha[C + (long long)dk * fnx * fny + (long long)dj * fnx + di];
        if (v == 0) zeros++;
        auto it = occur.find(v);
        if (it != occur.end())
          it->second++;
        else
          occur.insert({v, 1});
      }
  if (zeros > 0) return false;
  int n_alpha = 0, max_occ = 0;
  for (auto& it : occur) {
    n_alpha++;
    max_occ = std::max(max_occ, it.second);
  }
  if (n_alpha != 4 || max_occ > 10) return false;
  const long long plane = (long long)fnx * fny;
  std::fill(rec, rec + mNumNodeFeatures, -1);  // unused features stay -1
  rec[0] = (int)(C % fnx);
  rec[1] = (int)((C / fnx) % fny);
  rec[2] = (int)(C / plane);
  rec[3] = max_occ;
  int c = 0;
  for (auto& it : occur) rec[4 + c++] = it.first;
  return true;
}

void QOI3D::searchJunctionsOnImage(const QoiGrid& g, const int* alpha) {
  std::vector<int>& node = mQoIVectorIntData["node_region"];
  node.assign((size_t)40 * mNumActiveGrains * mNumNodeFeatures, -1);
  size_t node_cnt = 0;
  std::unordered_map<int, int> occur;
  int rec[9];
  for (int k = 1; k < g.fnz - 1; ++k)
    for (int j = 1; j < g.fny - 1; ++j)
      for (int i = 1; i < g.fnx - 1; ++i) {
        const long long C = (long long)k * g.fnx * g.fny + (long long)j * g.fnx + i;
        if (!junctionRecord(g, alpha, C, occur, rec)) continue;
        if ((node_cnt + 1) * mNumNodeFeatures > node.size()) continue;
        std::copy(rec, rec + mNumNodeFeatures, node.begin() + node_cnt * mNumNodeFeatures);
        node_cnt++;
      }
}

// The same records from the device's candidate list (ascending) and the
// per-cell distinct-value counts of the full scan.  The scan above reuses one
// hash map, cleared per cell; its bucket count only grows, with the largest
// number of values any earlier cell inserted, and fixes the order in which a
// record lists its grain ids.  Before each candidate the map is grown to the
// running maximum of those counts (filling it with that many keys and clearing
// it), so every record comes out as the full scan writes it.
void QOI3D::searchJunctionsOnCells(const QoiGrid& g, const int* alpha, const long long* cells,
                                   long long ncells, const unsigned char* distinct) {
  std::vector<int>& node = mQoIVectorIntData["node_region"];
  node.assign((size_t)40 * mNumActiveGrains * mNumNodeFeatures, -1);
  size_t node_cnt = 0;
  std::unordered_map<int, int> occur;
  int rec[9];
  const long long ni = g.fnx - 2, nj = g.fny - 2, plane = (long long)g.fnx * g.fny;
  long long scanned = 0;  // interior cells folded into running_max so far
  int running_max = 0, grown = 0;
  for (long long n = 0; n < ncells; ++n) {
    const long long C = cells[n];
    const long long k = C / plane, j = (C / g.fnx) % g.fny, i = C % g.fnx;
    const long long idx = (k - 1) * ni * nj + (j - 1) * ni + (i - 1);
    for (; scanned <= idx; ++scanned) running_max = std::max(running_max, (int)distinct[scanned]);
    if (running_max > grown) {
      occur.clear();
      for (int v = 0; v < running_max; ++v) occur.insert({v, 0});
      occur.clear();
      grown = running_max;
    }
    if (!junctionRecord(g, alpha, C, occur, rec)) continue;
    if ((node_cnt + 1) * mNumNodeFeatures > node.size()) continue;
    std::copy(rec, rec + mNumNodeFeatures, node.begin() + node_cnt * mNumNodeFeatures);
    node_cnt++;
  }
}

}  // namespace cupf_host
