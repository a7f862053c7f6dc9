"""parse_config / schema on the host (no GPU): the reference's config rules
(pichromatic-pipeline/src/config.rs:13-34, modules.rs)."""
import json

import pytest

IMGCONFIG_FILM = """
#### Pixel Pipeline ####
[[pipeline_modules]]
name = "Demosaic"
algorithm = "amaze"

[[pipeline_modules]]
name = "CFACoeffs"

[[pipeline_modules]]
name = "exp"            # names match case-insensitively
ev = 0

[[pipeline_modules]]
name = "CST"
target_color_space = { value = "AcesCg", description = "parameter form", choices = ["AcesCg"] }

[[pipeline_modules]]
name = "Film"
stock = "ColorNeg200"
film_format = "Film35mm"
seed = 1
output = "NegativeLinear"
"""


def test_parse_toml_config():
    from imops_b200.pipeline import parse_config
    assert parse_config(IMGCONFIG_FILM) is not None


def test_parse_json_config():
    from imops_b200.pipeline import parse_config
    cfg = {"pipeline_modules": [{"name": "Demosaic", "algorithm": "markesteijn"},
                                {"name": "CST", "target_color_space": "LinearSrgb"},
                                {"name": "Exp", "ev": {"value": 0.5, "description": "x"}}]}
    assert parse_config(json.dumps(cfg)) is not None


@pytest.mark.parametrize("text,msg", [
    ('[[pipeline_modules]]\nname = "Nope"\n', "wrong pipeline module name Nope"),
    ('[[pipeline_modules]]\nalgorithm = "amaze"\n', "Module must have a name field"),
    ('[[pipeline_modules]]\nname = "Exp"\n', "Invalid Exp config: missing field `ev`"),
    ('[[pipeline_modules]]\nname = "Demosaic"\nalgorithm = "AMaZE"\n', "unknown variant"),
    ('[[pipeline_modules]]\nname = "Film"\nstock = "X"\nfilm_format = "Film35mm"\nseed = 1\noutput = "NegativeLinear"\n',
     "Unknown film stock: X"),
    ('[[pipeline_modules]]\nname = "Film"\nstock = "BwStub"\nfilm_format = "Film35mm"\nseed = -1\n'
     'output = "NegativeLinear"\n', "seed"),
    ("this is not a config", "cant decode config from string"),
])
def test_config_errors(text, msg):
    from imops_b200 import ImopsError
    from imops_b200.pipeline import parse_config
    with pytest.raises(ImopsError) as e:
        parse_config(text)
    assert msg in e.value.message
    assert e.value.code == 9


def test_off_path_modules_parse():
    # modules that stay on the reference still parse with their field rules
    from imops_b200.pipeline import parse_config
    parse_config('[[pipeline_modules]]\nname = "BM3D"\nintensity = 0.5\n'
                 '[[pipeline_modules]]\nname = "LCH"\nlc = 1\ncc = 1\nhc = 1\n')


def test_schema_lists_modules_sorted_fields():
    from imops_b200.pipeline import get_pipeline_schema
    sch = get_pipeline_schema()
    names = [m["name"] for m in sch]
    assert names[:4] == ["Demosaic", "ChromaDenoise", "LumaGuidedChromaDenoise", "CFACoeffs"]
    film = next(m for m in sch if m["name"] == "Film")
    assert [f["name"] for f in film["fields"]] == ["film_format", "output", "seed", "stock"]
    seed = next(f for f in film["fields"] if f["name"] == "seed")
    assert seed["field_type"] == "integer" and seed["default_value"] == 1
    dem = sch[0]["fields"][0]
    assert dem["default_value"] == "amaze" and "markesteijn" in dem["choices"]
    exp = next(m for m in sch if m["name"] == "Exp")
    assert exp["fields"][0]["field_type"] == "float"
