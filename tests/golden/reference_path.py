"""Where the fixture recipe finds the reference's checkout (read-only): the
MEEP_TORCH_REF environment variable, else the checkout this build was made beside."""
import os

REF = os.environ.get("MEEP_TORCH_REF", "/root/reference")
