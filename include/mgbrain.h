// Umbrella header of the MGBrain C++ API (same typedefs as the reference's
// src/mgbrain.h:11-31), backed by the mgbrain_b200 CUDA core.
#pragma once
#include "mgbrain/constgen.h"
#include "mgbrain/macro.h"
#include "mgbrain/maker.h"
#include "mgbrain/mgsim.h"
#include "mgbrain/model.h"
#include "mgbrain/netgen.h"
#include "mgbrain/network.h"
#include "mgbrain/parser.h"
#include "mgbrain/parter.h"

typedef MGBrain::Config config;
typedef MGBrain::Model model;
typedef MGBrain::Population pop;
typedef MGBrain::Projection prj;
typedef MGBrain::Network network;
typedef MGBrain::NeuronType neuType;
typedef MGBrain::Neuron neuron;
typedef MGBrain::Synapse synapse;
typedef MGBrain::NetGen netgen;
typedef MGBrain::Partitioner parter;
typedef MGBrain::PartType PartType;
typedef MGBrain::MGSimulator mgsim;
typedef MGBrain::NeuronType NeuType;
typedef MGBrain::real real;
typedef MGBrain::PartitionAnalysis panalysis;
typedef MGBrain::ConstGen constgen;
typedef MGBrain::ModelMaker maker;
typedef MGBrain::ParamsParser parser;
typedef MGBrain::timer timer;
