};  // struct RefHighlights
}  // namespace libraw_enhanced

/* C ABI over the streamed member function.  rgb is (H, W, 3) float, updated
 * in place; mask_out (W*H floats) and wb_rgb (3 floats) may be null.  The
 * reference returns its highlight max as a bool; *max_val_out gets 1 or 0.
 * std::cout is muted for the call unless LRE_REF_VERBOSE is set. */
extern "C" int ref_recover_highlights(float* rgb, size_t w, size_t h, float saturation_threshold,
                                      float* mask_out, const float* wb_rgb) {
  std::streambuf* saved = nullptr;
  if (!std::getenv("LRE_REF_VERBOSE")) saved = std::cout.rdbuf(nullptr);
  libraw_enhanced::ImageBufferFloat buf;
  buf.image = reinterpret_cast<float (*)[3]>(rgb);
  buf.width = w;
  buf.height = h;
  buf.channels = 3;
  libraw_enhanced::RefHighlights r;
  const bool ok = r.recover_highlights(buf, saturation_threshold, mask_out, wb_rgb);
  if (saved) {
    std::cout.rdbuf(saved);
    std::cout.clear();
  }
  return ok ? 1 : 0;
}
