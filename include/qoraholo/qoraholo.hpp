#pragma once

#include "qoraholo/array.hpp"
#include "qoraholo/backend.hpp"
#include "qoraholo/bpm.hpp"
#include "qoraholo/field.hpp"
#include "qoraholo/odt.hpp"
#include "qoraholo/phantom.hpp"
#include "qoraholo/pipeline.hpp"
#include "qoraholo/unwrap.hpp"
