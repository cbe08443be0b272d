// Differentiable layer interface (src/layers/layer.h:19-70).
// Ownership: input and grad_output are borrowed, output and grad_input owned.
#pragma once

class Layer {
 public:
  virtual ~Layer() = default;
  virtual void forward() = 0;
  virtual void backward() = 0;
  virtual void zeroGrad() = 0;
};

template <typename TIn, typename TOut, typename TGradIn, typename TGradOut>
class TypedLayer : public Layer {
 public:
  void setInput(const TIn* in_) { input = in_; }
  TOut& getOutput() { return output; }
  void setGradOutput(const TGradOut* gout_) { grad_output = gout_; }
  TGradIn& getGradInput() { return grad_input; }

  virtual void allocate(int n) { output.allocate(n); }
  virtual void allocateGrad(int n) { grad_input.allocate(n); }
  void zeroGrad() override { grad_input.zero(); }

 protected:
  const TIn* input = nullptr;
  TOut output;
  const TGradOut* grad_output = nullptr;
  TGradIn grad_input;
};
