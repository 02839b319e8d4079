// label_oracle.cpp -- CPU restatement of Connect (DPE.cpp:27-134), the labelling EdgeSegment
// applies to its binary maps (DPE.cpp:160-162, 255-256).
//
// TEST INFRASTRUCTURE ONLY: the checker for the device labelling and for the host preprocessing's
// vectorised form.  A literal restatement of the reference loop: provisional labels in raster
// order, a join of two different labels recorded as connection[larger] = smaller (overwriting an
// earlier join of the same label, which the reference then loses), chain ends as final labels,
// renumbered in increasing order.  PARITY UNPINNED against the reference itself (which needs
// OpenCV to build); checked against a pure-Python restatement of the same lines in the tests.
#include <cstdint>
#include <vector>

extern "C" int oracle_connect(const uint8_t *img, int cols, int rows, int32_t *labels, int32_t *counts,
                              int counts_capacity, int *num_labels) {
  if (!img || !labels || cols < 1 || rows < 1) return 1;
  std::vector<int> lab((size_t)rows * cols, 0);
  std::vector<int> connection(1, 0);
  int cnt = 1;
  for (int y = 0; y < rows; ++y)
    for (int x = 0; x < cols; ++x) {
      const size_t p = (size_t)y * cols + x;
      if (img[p] == 255) {
        lab[p] = 0;
        continue;
      }
      const bool left = x > 0 && img[p] == 0 && img[p - 1] == 0;
      const bool up = y > 0 && img[p] == 0 && img[p - cols] == 0;
      if (left) lab[p] = lab[p - 1];
      if (up) lab[p] = lab[p - cols];
      if (!left && !up) {
        lab[p] = cnt;
        connection.push_back(cnt);
        cnt++;
      } else if (left && up) {
        const int l = lab[p - 1], u = lab[p - cols];
        if (l > u) {
          connection[l] = u;
          lab[p] = lab[p - cols];
        } else if (l < u) {
          connection[u] = l;
          lab[p] = lab[p - 1];
        }
      }
    }
  for (size_t i = 1; i < connection.size(); ++i) {
    int cur = connection[i], pre = connection[cur];
    while (pre != cur) {
      cur = pre;
      pre = connection[pre];
    }
    connection[i] = cur;
  }
  int label_num = 1;
  std::vector<int> mapping(connection.size(), 0);
  for (size_t i = 1; i < connection.size(); ++i)
    if (connection[i] == (int)i) mapping[i] = label_num++;
  for (size_t i = 1; i < connection.size(); ++i) connection[i] = mapping[connection[i]];
  for (int k = 0; k < counts_capacity && counts; ++k) counts[k] = 0;
  for (size_t p = 0; p < (size_t)rows * cols; ++p) {
    const int l = connection[lab[p]];
    labels[p] = l;
    if (counts && l < counts_capacity) counts[l]++;
  }
  if (num_labels) *num_labels = label_num;
  return label_num > counts_capacity ? 2 : 0;
}
