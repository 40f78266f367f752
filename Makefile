# Build of the tensorsvm B200 library (sm_100a), the CLI and the oracle's C part.
#   make            -> tensorsvm_b200/lib/libtensorsvm_b200.so, tensorsvm_b200/bin/tensorsvm-train,
#                      tensorsvm_b200/bin/tensorsvm-predict
#   make oracle     -> oracle/_build/liboracle_sketch.so
#   make reference  -> oracle/_ref/tensorsvm-train-ref (needs the reference source)
NVCC      ?= nvcc
CUDA_HOME ?= /usr/local/cuda
ARCH      := -gencode arch=compute_100a,code=sm_100a
NVFLAGS   := -O3 -std=c++17 $(ARCH) -lineinfo -Xcompiler -fPIC -Iinclude -Itensorsvm_b200/csrc \
             --expt-relaxed-constexpr -Xptxas -warn-spills
CSRC      := $(wildcard tensorsvm_b200/csrc/*.cu)
CPPSRC    := $(wildcard tensorsvm_b200/csrc/*.cpp)
OBJDIR    := tensorsvm_b200/_build
OBJS      := $(patsubst tensorsvm_b200/csrc/%.cu,$(OBJDIR)/%.o,$(CSRC)) \
             $(patsubst tensorsvm_b200/csrc/%.cpp,$(OBJDIR)/%.host.o,$(CPPSRC))
LIB       := tensorsvm_b200/lib/libtensorsvm_b200.so
CLI       := tensorsvm_b200/bin/tensorsvm-train
PREDICT   := tensorsvm_b200/bin/tensorsvm-predict
HDRS      := $(wildcard tensorsvm_b200/csrc/*.h tensorsvm_b200/csrc/*.cuh) include/tensorsvm.h

all: $(LIB) $(CLI) $(PREDICT)

$(OBJDIR)/%.o: tensorsvm_b200/csrc/%.cu $(HDRS)
	@mkdir -p $(OBJDIR)
	$(NVCC) $(NVFLAGS) -c $< -o $@

$(OBJDIR)/%.host.o: tensorsvm_b200/csrc/%.cpp include/tensorsvm.h tensorsvm_b200/csrc/trace.h
	@mkdir -p $(OBJDIR)
	g++ -O3 -std=c++17 -fPIC -pthread -Wall -Iinclude -I$(CUDA_HOME)/include -c $< -o $@

$(LIB): $(OBJS)
	@mkdir -p $(dir $@)
	$(NVCC) $(ARCH) -shared -o $@ $(OBJS) -lcudart -Xcompiler -pthread

$(CLI): tensorsvm_b200/cli/tensorsvm_train.cpp include/tensorsvm.h $(LIB)
	@mkdir -p $(dir $@)
	g++ -O2 -std=c++17 -Iinclude $< -o $@ -Ltensorsvm_b200/lib -ltensorsvm_b200 \
	    -Wl,-rpath,'$$ORIGIN/../lib'

$(PREDICT): tensorsvm_b200/cli/tensorsvm_predict.cpp include/tensorsvm.h $(LIB)
	@mkdir -p $(dir $@)
	g++ -O2 -std=c++17 -Iinclude $< -o $@ -Ltensorsvm_b200/lib -ltensorsvm_b200 \
	    -Wl,-rpath,'$$ORIGIN/../lib'

oracle:
	python3 -c "from oracle import oracle; oracle.build(force=True)"

reference:
	bash oracle/build_ref.sh

clean:
	rm -rf $(OBJDIR) tensorsvm_b200/lib tensorsvm_b200/bin

.PHONY: all oracle reference clean
