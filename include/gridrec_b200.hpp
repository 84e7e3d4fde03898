// gridrec_b200.hpp -- header-only C++ class with the reference's GridRec call
// surface (gridrec/GPU/gridrec.h:72-143, gridrec/GPU/recon_algorithm.h:56-95)
// implemented on the C ABI of gridrec_b200.h.
//
// Drop-in use from the reference's callers (tomo_recon.cpp:1701-1706,
// 3846-3852; find_shift.cpp:1661-1666, 1836-1841): replace `GridRec` by
// `gridrec_b200::GridRec`; the setter sequence, the host buffers (sinogram
// n_ang x n_det float, reconstruction n_det rows of n_det floats with the
// leading M0 x M0 block written) and the two-slices-per-call contract stay.
// Differences, all additive: setCenter() (GridRec::init fixes n_det/2,
// gridrec.cu:227), setCenterShift() of find_shift's GridRec (centre = n_det/2 +
// shift, find_shift/src/main/gridrec.cu:229, 809-813), lastStatus() instead of
// exit(2) on bad parameters, and no cuFFT or cutil dependency.
#ifndef GRIDREC_B200_HPP
#define GRIDREC_B200_HPP

#include <cstring>
#include <vector>

#include "gridrec_b200.h"

namespace gridrec_b200 {

class GridRec {
 public:
  GridRec() = default;
  ~GridRec() { destroy(); }
  GridRec(const GridRec&) = delete;
  GridRec& operator=(const GridRec&) = delete;

  int numberOfSinogramsNeeded() const { return 2; }
  int numberOfReconstructions() const { return 2; }

  void setSinogramDimensions(int x_dim, int y_dim) {
    n_det_ = x_dim;
    n_ang_ = y_dim;
  }
  int getSinogramXDimension() const { return n_det_; }
  int getSinogramYDimension() const { return n_ang_; }

  // The reference keeps the pointer and reads it in init(); so does this class.
  void setThetaList(float* theta_list, int theta_list_size) {
    theta_ = theta_list;
    n_theta_ = theta_list_size;
  }
  int getThetaListSize() const { return n_theta_; }
  float* getThetaList() const { return theta_; }

  void setFilter(int filter_name) { filter_ = filter_name; }
  int getFilter() const { return filter_; }
  void setGPUDeviceID(int id) { device_ = id; }
  int getGPUDeviceID() const { return device_; }
  void setCenter(float center) {
    center_ = center;
    shift_set_ = false;
  }
  // find_shift's GridRec: the centre is n_det / 2 (integer division) + shift,
  // applied at init() (find_shift/src/main/gridrec.cu:229, 809-813)
  void setCenterShift(float shift) {
    shift_ = shift;
    shift_set_ = true;
  }
  float getCenter() const { return shift_set_ ? (float)(n_det_ / 2) + shift_ : center_; }

  void init() {
    destroy();
    gr_params p;
    gr_params_default(&p, n_det_, n_ang_, theta_);
    p.center = getCenter();
    p.filter = filter_;
    p.device = device_;
    status_ = gr_plan_create(&p, &plan_);
    if (status_ == GR_OK) gr_plan_sizes(plan_, nullptr, nullptr, &m0_, nullptr, nullptr);
  }

  void setSinoAndReconBuffers(int number, float* sinogram, float* reconstruction) {
    if (number == 1) {
      sino_[0] = sinogram;
      recon_[0] = reconstruction;
    } else if (number == 2) {
      sino_[1] = sinogram;
      recon_[1] = reconstruction;
    }
  }

  // Reconstructs both slices into the reconstruction buffers (host memory,
  // row stride n_det, M0 x M0 block), as GridRec::reconstruct (gridrec.cu:314).
  void reconstruct() {
    if (!plan_ || !sino_[0] || !recon_[0]) {
      status_ = GR_ERR_ARG;
      return;
    }
    if (m0_ <= n_det_) {  // the caller's buffers directly (power-of-two widths: M0 = n_det - 1)
      status_ = gr_reconstruct_pair_host(plan_, sino_[0], sino_[1], recon_[0], recon_[1], n_det_,
                                         nullptr);
      return;
    }
    // M0 > n_det (other widths): the reference's rows of stride n_det overlap
    // (gridrec.cu:196-197); here the images go through a staging buffer and each
    // row keeps its first n_det values
    const size_t slice = (size_t)n_ang_ * n_det_;
    in_.resize(2 * slice);
    std::memcpy(in_.data(), sino_[0], slice * sizeof(float));
    if (sino_[1]) std::memcpy(in_.data() + slice, sino_[1], slice * sizeof(float));
    else std::memset(in_.data() + slice, 0, slice * sizeof(float));
    const long stride = n_det_ > m0_ ? n_det_ : m0_;
    out_.assign(2 * (size_t)m0_ * stride, 0.f);
    gr_batch_desc b;
    std::memset(&b, 0, sizeof(b));
    b.n_slices = 2;
    b.dtype = GR_DTYPE_F32;
    b.sinos = in_.data();
    b.outs = out_.data();
    b.out_stride = stride;
    status_ = gr_reconstruct_host(plan_, &b, nullptr);
    if (status_ != GR_OK) return;
    for (int s = 0; s < 2; ++s) {
      if (!recon_[s]) continue;
      const float* src = out_.data() + (size_t)s * m0_ * stride;
      for (int j = 0; j < m0_; ++j)
        std::memcpy(recon_[s] + (size_t)j * n_det_, src + (size_t)j * stride,
                    (size_t)(m0_ < n_det_ ? m0_ : n_det_) * sizeof(float));
    }
  }

  void destroy() {
    if (plan_) gr_plan_destroy(plan_);
    plan_ = nullptr;
  }

  int imageSize() const { return m0_; }   // M0 (GridRec's imgsiz)
  int lastStatus() const { return status_; }
  const char* lastError() const { return gr_last_error(); }

 private:
  int n_det_ = 0, n_ang_ = 0, n_theta_ = 0, filter_ = GR_FILTER_NONE, device_ = 0, m0_ = 0;
  float center_ = -1.f, shift_ = 0.f;
  bool shift_set_ = false;
  float* theta_ = nullptr;
  float* sino_[2] = {nullptr, nullptr};
  float* recon_[2] = {nullptr, nullptr};
  gr_plan* plan_ = nullptr;
  int status_ = GR_OK;
  std::vector<float> in_, out_;
};

}  // namespace gridrec_b200

#endif  // GRIDREC_B200_HPP
